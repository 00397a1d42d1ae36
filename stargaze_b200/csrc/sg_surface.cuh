// sg_surface.cuh — the procedural surface styles 1-6 of surface_albedo
// (pathtrace.wgsl:357-910): gas giant, cratered, rocky, icy, volcanic and
// terran bodies, each a function of the body-local normal and the body's
// pattern parameters (axis_y.w seed, surface_color, surface_params).
//
// The patterns hash lattice coordinates through fract() of large products
// (hash31), which turns any last-bit difference of a coordinate into a
// visibly different value. So every operation here is IEEE single
// precision with no contraction (the `sf` and `sv` types below wrap the
// round-to-nearest intrinsics), and sines, cosines, arc tangents,
// exponentials and powers are evaluated in double and rounded to float:
// the correctly rounded value, which the CPU restatement computes the same
// way. The style code runs only where a styled body is shaded, out of line.
#pragma once

#include "sg_device.cuh"

namespace sg {

namespace style {

// A float whose arithmetic is never fused or reassociated.
struct sf {
    float v;
    __device__ __forceinline__ sf() : v(0.0f) {}
    __device__ __forceinline__ sf(float x) : v(x) {}
};
__device__ __forceinline__ sf operator+(sf a, sf b) { return sf(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ sf operator-(sf a, sf b) { return sf(__fsub_rn(a.v, b.v)); }
__device__ __forceinline__ sf operator*(sf a, sf b) { return sf(__fmul_rn(a.v, b.v)); }
__device__ __forceinline__ sf operator/(sf a, sf b) { return sf(__fdiv_rn(a.v, b.v)); }
__device__ __forceinline__ sf operator-(sf a) { return sf(-a.v); }
__device__ __forceinline__ sf &operator+=(sf &a, sf b) { return a = a + b; }
__device__ __forceinline__ sf &operator-=(sf &a, sf b) { return a = a - b; }
__device__ __forceinline__ sf &operator*=(sf &a, sf b) { return a = a * b; }
__device__ __forceinline__ bool operator<(sf a, sf b) { return a.v < b.v; }
__device__ __forceinline__ bool operator>(sf a, sf b) { return a.v > b.v; }
__device__ __forceinline__ bool operator<=(sf a, sf b) { return a.v <= b.v; }
__device__ __forceinline__ bool operator>=(sf a, sf b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator==(sf a, sf b) { return a.v == b.v; }

__device__ __forceinline__ sf floorf(sf a) { return sf(::floorf(a.v)); }
__device__ __forceinline__ sf sqrtf(sf a) { return sf(__fsqrt_rn(a.v)); }
__device__ __forceinline__ sf fabsf(sf a) { return sf(::fabsf(a.v)); }
__device__ __forceinline__ sf minf_(sf a, sf b) { return a < b ? a : b; }
__device__ __forceinline__ sf maxf_(sf a, sf b) { return a > b ? a : b; }
__device__ __forceinline__ sf clampf_(sf x, sf lo, sf hi) { return minf_(maxf_(x, lo), hi); }
__device__ __forceinline__ sf mixf(sf a, sf b, sf t) { return a * (sf(1.0f) - t) + b * t; }
__device__ __forceinline__ sf smoothstepf(sf e0, sf e1, sf x) {
    const sf t = clampf_((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (sf(3.0f) - sf(2.0f) * t);
}
__device__ __forceinline__ sf stepf(sf edge, sf x) { return x >= edge ? sf(1.0f) : sf(0.0f); }
// Correctly rounded transcendentals (double, then one rounding).
__device__ __forceinline__ sf sin_d(sf x) { return sf((float)::sin((double)x.v)); }
__device__ __forceinline__ sf cos_d(sf x) { return sf((float)::cos((double)x.v)); }
__device__ __forceinline__ sf atan2_d(sf y, sf x) { return sf((float)::atan2((double)y.v, (double)x.v)); }
__device__ __forceinline__ sf exp_d(sf x) { return sf((float)::exp((double)x.v)); }
__device__ __forceinline__ sf pow_d(sf x, sf y) { return sf((float)::pow((double)x.v, (double)y.v)); }
__device__ __forceinline__ sf surface_gaussian(sf distance) { return exp_d(-(distance * distance)); }
__device__ __forceinline__ sf ridge(sf n, sf width) { return sf(1.0f) - smoothstepf(0.0f, width, fabsf(n - sf(0.5f))); }

constexpr float PI_F = 3.141592653589793f;
constexpr float TAU_F = 6.283185307179586f;

// A vector of such floats.
struct sv {
    sf x, y, z;
};
__device__ __forceinline__ sv V(sf x, sf y, sf z) { return sv{x, y, z}; }
__device__ __forceinline__ sv xyzs(float4 v) { return V(v.x, v.y, v.z); }
__device__ __forceinline__ float3 to_f3(sv a) { return f3(a.x.v, a.y.v, a.z.v); }
__device__ __forceinline__ sv vadd(sv a, sv b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ sv vsub(sv a, sv b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ sv vmul(sv a, sf s) { return V(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ sv vmulv(sv a, sv b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ sv vdivs(sv a, sf s) { return V(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ sv vadds(sv a, sf s) { return V(a.x + s, a.y + s, a.z + s); }
__device__ __forceinline__ sv vsubs(sv a, sf s) { return V(a.x - s, a.y - s, a.z - s); }
__device__ __forceinline__ sf vdot(sv a, sv b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ sv vcross(sv a, sv b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ sf vlength(sv a) { return sqrtf(vdot(a, a)); }
__device__ __forceinline__ sv vnormalize(sv a) {
    const sf inv = sf(1.0f) / sqrtf(vdot(a, a));
    return vmul(a, inv);
}
__device__ __forceinline__ sv vmix(sv a, sv b, sf t) { return V(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }
__device__ __forceinline__ sv vfloor(sv a) { return V(floorf(a.x), floorf(a.y), floorf(a.z)); }
// The value noise of surface_albedo (strict already).
__device__ __forceinline__ sf hash31(sv p) { return sf(sg::hash31(to_f3(p))); }
__device__ __forceinline__ sf vnoise(sv p) { return sf(sg::vnoise(to_f3(p))); }


/* fbm: pathtrace.wgsl:357-373 (the octave rotation is a column matrix). */
static __device__ __noinline__ sf fbm(sv p, uint32_t octaves) {
    sf amplitude = 0.5f, sum = 0.0f, norm = 0.0f;
    for (uint32_t octave = 0; octave < octaves; octave++) {
        sum += amplitude * vnoise(p);
        norm += amplitude;
        sv r = V((0.0f * p.x + -1.6f * p.y) + -1.2f * p.z, (1.6f * p.x + 0.72f * p.y) + -0.96f * p.z,
                 (1.2f * p.x + -0.96f * p.y) + 1.28f * p.z);
        p = vadd(r, V(17.3f, 5.1f, 11.7f));
        amplitude *= 0.5f;
    }
    return sum / norm;
}
/* seed_offset: pathtrace.wgsl:384-389 */
static __device__ __noinline__ sv seed_offset(sf seed) {
    return vmul(V(hash31(V(seed, 1.0f, 7.0f)), hash31(V(3.0f, seed, 5.0f)), hash31(V(9.0f, 2.0f, seed))), 512.0f);
}

/* gas_giant_albedo: pathtrace.wgsl:394-472 */
static __device__ __noinline__ sv gas_giant_albedo(const float4 *body, sv local) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sv zone = xyzs(body[kMaterial]), belt = xyzs(body[kSurfaceColor]);
    sf turbulence = sf(body[kSurfaceColor].w);
    sf bands = sf(body[kSurfaceParams].x);
    uint32_t storms = (uint32_t)(body[kSurfaceParams].y + 0.5f);
    sv q = local;
    sf masks[3] = {0, 0, 0}, rims[3] = {0, 0, 0};
    for (uint32_t k = 0; k < storms && k < 3u; k++) {
        sf fk = (float)k;
        sf lat = (hash31(vadd(off, V(7.1f * fk, 1.3f, 2.9f))) - 0.5f) * 1.1f;
        sf lon = hash31(vadd(off, V(3.7f, 5.3f * fk, 8.1f))) * TAU_F;
        sf size = (k == 0u ? 0.11f : 0.05f) * (0.8f + 0.4f * hash31(vadd(off, V(fk, 9.0f, 4.0f))));
        sv centre = V(cos_d(lat) * cos_d(lon), cos_d(lat) * sin_d(lon), sin_d(lat));
        if (vdot(q, centre) <= 0.0f) continue;
        sv east = V(-sin_d(lon), cos_d(lon), 0.0f);
        sv north = vcross(centre, east);
        sf dx = vdot(vsub(q, centre), east) / (2.0f * size);
        sf dy = vdot(vsub(q, centre), north) / size;
        sf e = sqrtf(dx * dx + dy * dy);
        sf influence = 1.0f - smoothstepf(0.0f, 2.4f, e);
        sf angle = (lat < 0.0f ? 3.2f : -3.2f) * influence * influence;
        sf c = cos_d(angle), s = sin_d(angle);
        sf rx = c * dx - s * dy;
        sf ry = s * dx + c * dy;
        q = vnormalize(vadd(vadd(q, vmul(east, (rx - dx) * 2.0f * size)), vmul(north, (ry - dy) * size)));
        sf ragged = e + 0.25f * (fbm(vadd(vmul(q, 18.0f), off), 3) - 0.5f);
        masks[k] = 1.0f - smoothstepf(0.7f, 1.0f, ragged);
        rims[k] = smoothstepf(0.75f, 1.0f, ragged) * (1.0f - smoothstepf(1.0f, 1.35f, ragged));
    }
    sv p = vadd(V(q.x * 2.2f, q.y * 2.2f, q.z * 9.0f), off);
    sf warp1 = fbm(p, 5) - 0.5f;
    sf warp2 = fbm(vadds(vadd(vmul(p, 2.1f), V(5.2f, 1.3f, 7.7f)), 4.0f * warp1), 5) - 0.5f;
    sf lat = q.z + 0.07f * sin_d(3.0f * PI_F * q.z + off.z) + 0.04f * sin_d(5.0f * PI_F * q.z + off.y);
    sf shear = 0.35f + 0.65f * fabsf(cos_d(PI_F * bands * lat + off.x));
    sf lon = atan2_d(q.y, q.x);
    sf ripple = sin_d(lon * (9.0f + floorf(bands)) + 6.0f * warp1 + off.y) * 0.5f +
                   sin_d(lon * 23.0f + 9.0f * warp2 + off.z) * 0.25f;
    sf mu = lat + turbulence * shear * (0.16f * warp1 + 0.10f * warp2 + 0.025f * ripple);
    sf wave = 0.5f + 0.5f * sin_d(PI_F * bands * mu + off.x);
    sf irregular = fbm(V(mu * bands * 1.7f, off.y, off.z), 3);
    sf profile = 0.5f * wave + 0.5f * irregular;
    sf tone = fbm(V(mu * bands * 0.9f, off.z, off.x), 2);
    sf fine = fbm(vadds(vadd(V(q.x * 7.0f, q.y * 7.0f, q.z * 70.0f), off), 3.0f * warp2), 4);
    sf eddies = fbm(vadd(vmul(p, 5.0f), vmul(V(warp1, warp2, warp1), 6.0f)), 4);
    sv color = vmix(belt, zone, smoothstepf(0.3f, 0.75f, profile));
    color = vmix(color, vmulv(color, vadds(vmul(color, 0.5f), 0.55f)), smoothstepf(0.35f, 0.75f, tone) * 0.8f);
    color = vmul(color, (0.78f + 0.44f * fine) * (0.9f + 0.2f * eddies));
    sf polar = smoothstepf(0.55f, 0.92f, fabsf(local.z));
    color = vmix(color, vmul(vmix(zone, belt, 0.55f), 0.8f + 0.2f * fine), polar * 0.8f);
    for (uint32_t k = 0; k < storms && k < 3u; k++) {
        sv tint = k == 0u ? vmul(vmulv(belt, belt), 1.5f) : vmul(zone, 1.15f);
        sf core = 1.0f - 0.25f * (1.0f - smoothstepf(0.0f, 0.6f, masks[k] - rims[k]));
        color = vmix(color, vmul(vmul(tint, 0.7f + 0.6f * fine), core), masks[k] * 0.92f);
        color = vmix(color, vmul(zone, 1.1f), rims[k] * 0.45f);
    }
    return color;
}

/* surface_gaussian, hash33, ridge, maria, cell_centre: pathtrace.wgsl:477-516 */
static __device__ __noinline__ sv hash33(sv p) {
    return V(hash31(p), hash31(vadd(p, V(19.1f, 7.3f, 3.7f))), hash31(vadd(p, V(5.9f, 31.7f, 11.3f))));
}
static __device__ __noinline__ sf maria(sv q, sv off) {
    sf warp = fbm(vadd(vmul(q, 2.0f), off), 4) - 0.5f;
    return smoothstepf(0.5f, 0.56f, fbm(vadds(vadd(vmul(q, 1.2f), off), 1.5f * warp), 5));
}
__device__ __forceinline__ int cell_centre(sv cell, sv key, sf scale, sv off, sv *centre_out) {
    for (uint32_t t = 0; t < 3u; t++) {
        sv centre = vnormalize(vsub(vadd(cell, hash33(vadds(key, (float)t * 17.0f))), off));
        sv f = vfloor(vadd(vmul(centre, scale), off));
        if (f.x == cell.x && f.y == cell.y && f.z == cell.z) {
            *centre_out = centre;
            return 1;
        }
    }
    return 0;
}
__device__ __forceinline__ sv corner(sv base, uint32_t i) {
    return vadd(base, V((float)(i & 1u), (float)((i >> 1u) & 1u), (float)((i >> 2u) & 1u)));
}

/* crater_layer: pathtrace.wgsl:527-633. state = (floor darkness, relief). */
static __device__ __noinline__ void crater_layer(sv q, sf scale, sf density, sv off, sv body_off, sf flood, sf contrast,
                         sf rays, sf state[2]) {
    sv p = vadd(vmul(q, scale), off);
    sv base = vfloor(vsubs(p, 0.5f));
    uint32_t slots[6];
    sf ages[6];
    sv centres[6];
    uint32_t count = 0;
    for (uint32_t i = 0; i < 16u; i++) {
        sv grid = corner(base, i);
        sv a = vsub(grid, p), b = vsubs(vsub(p, grid), 1.0f);
        sv gap = V(maxf_(maxf_(a.x, b.x), 0.0f), maxf_(maxf_(a.y, b.y), 0.0f), maxf_(maxf_(a.z, b.z), 0.0f));
        if (vdot(gap, gap) > 0.2343f) continue;
        sv key = vadds(grid, (float)(i >> 3u) * 1000.0f);
        if (hash31(vadd(key, V(71.3f, 3.1f, 9.7f))) > density) continue;
        sv found;
        if (!cell_centre(grid, key, scale, off, &found)) continue;
        sf size = hash31(vadd(key, V(3.1f, 8.3f, 1.7f)));
        sf radius = (0.06f + 0.16f * size * size) / scale;
        if (vlength(vsub(q, found)) > 2.2f * radius) continue;
        sf age = hash31(vadd(key, V(29.0f, 61.0f, 7.0f)));
        if (flood > 0.0f && age < 0.7f && maria(found, body_off) > 0.5f) continue;
        if (count == 6u) {
            if (age <= ages[0]) continue;
            for (uint32_t m = 0; m < 5u; m++) {
                ages[m] = ages[m + 1];
                slots[m] = slots[m + 1];
                centres[m] = centres[m + 1];
            }
            count = 5u;
        }
        uint32_t j = count;
        while (j > 0u && ages[j - 1] > age) {
            ages[j] = ages[j - 1];
            slots[j] = slots[j - 1];
            centres[j] = centres[j - 1];
            j--;
        }
        ages[j] = age;
        slots[j] = i;
        centres[j] = found;
        count++;
    }
    sf floor_shade = 1.0f, relief = state[1];
    for (uint32_t k = 0; k < count; k++) {
        uint32_t i = slots[k];
        sv cell = vadds(corner(base, i), (float)(i >> 3u) * 1000.0f);
        sv centre = centres[k];
        sf size = hash31(vadd(cell, V(3.1f, 8.3f, 1.7f)));
        sf radius = (0.06f + 0.16f * size * size) / scale;
        sv offset = vsub(q, centre);
        sf d = vlength(offset) / radius;
        sv east = vcross(V(0.0f, 0.0f, 1.0f), centre);
        east = vdivs(east, maxf_(vlength(east), 1.0e-4f));
        sv north = vcross(centre, east);
        sf angle = atan2_d(vdot(offset, north), vdot(offset, east));
        sv phase = vmul(hash33(vadd(cell, V(41.0f, 5.0f, 23.0f))), TAU_F);
        sf wobble = 0.025f * (sin_d(3.0f * angle + phase.x) + sin_d(5.0f * angle + phase.y) +
                                 0.6f * sin_d(8.0f * angle + phase.z));
        sf r = d + wobble;
        floor_shade = minf_(floor_shade, 1.0f - 0.18f * contrast * (1.0f - smoothstepf(0.55f, 0.9f, r)));
        sf rim = 0.22f * contrast * surface_gaussian((r - 1.0f) / 0.13f);
        sf footprint = 1.0f - smoothstepf(1.1f, 1.3f, r);
        relief = mixf(relief, rim, footprint);
        sf blanket = (1.0f - smoothstepf(1.0f, 1.9f, r)) * (1.0f - footprint);
        relief = mixf(relief, 0.0f, blanket * 0.3f) + 0.1f * contrast * blanket;
        sf fresh = hash31(vadd(cell, V(13.0f, 2.0f, 5.0f)));
        if (rays > 0.0f && fresh > 0.82f) {
            sf streaks = pow_d(vnoise(V(cos_d(angle) * 9.0f, sin_d(angle) * 9.0f, fresh * 40.0f)), 3.0f);
            relief += contrast * (rays * 0.9f * streaks * (1.0f - smoothstepf(1.0f, 2.2f, d)) * stepf(0.9f, d) +
                                  rays * 0.25f * (1.0f - smoothstepf(0.0f, 1.0f, d)));
        }
    }
    state[0] *= floor_shade;
    state[1] = relief;
}

/* craters: pathtrace.wgsl:636-647 */
static __device__ __noinline__ sf craters(sv q, sf density, sv off, sf flood, sf contrast, sf rays) {
    if (density <= 0.0f) return 1.0f;
    sf state[2] = {1.0f, 0.0f};
    crater_layer(q, 1.5f, density, off, off, flood, contrast, rays, state);
    crater_layer(q, 3.5f, density, vadds(off, 101.0f), off, flood, contrast, rays * 0.8f, state);
    crater_layer(q, 8.0f, density, vadds(off, 203.0f), off, flood, contrast * 0.85f, rays * 0.5f, state);
    crater_layer(q, 18.0f, density, vadds(off, 307.0f), off, 0.0f, contrast * 0.7f, 0.0f, state);
    crater_layer(q, 40.0f, density, vadds(off, 401.0f), off, 0.0f, contrast * 0.55f, 0.0f, state);
    return state[0] * (1.0f + state[1]);
}

/* polar_caps: pathtrace.wgsl:650-656 */
static __device__ __noinline__ sf polar_caps(sv q, sf extent, sv off) {
    if (extent <= 0.0f) return 0.0f;
    sf edge = 1.0f - extent + 0.12f * (fbm(vadd(vmul(q, 5.0f), off), 5) - 0.5f) +
                 0.05f * (fbm(vadd(vmul(q, 18.0f), off), 3) - 0.5f);
    return smoothstepf(edge - 0.015f, edge + 0.015f, fabsf(q.z));
}

/* cratered_albedo: pathtrace.wgsl:660-669 */
static __device__ __noinline__ sv cratered_albedo(const float4 *body, sv q) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sf mare = maria(q, off);
    sf grain = fbm(vadd(vmul(q, 45.0f), off), 3);
    sv color = vmix(xyzs(body[kMaterial]), xyzs(body[kSurfaceColor]), mare);
    color = vmul(color, 0.9f + 0.2f * grain);
    return vmul(color, craters(q, sf(body[kSurfaceColor].w), off, 1.0f, 1.0f, 1.0f));
}

/* rocky_albedo: pathtrace.wgsl:673-687 */
static __device__ __noinline__ sv rocky_albedo(const float4 *body, sv q) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sv base = vadd(vmul(q, 1.8f), off);
    sv warp = vsubs(V(fbm(base, 4), fbm(vadds(base, 7.0f), 4), 0.0f), 0.5f);
    sf dark = smoothstepf(0.5f, 0.64f, fbm(vadd(vadd(vmul(q, 2.2f), off), V(2.0f * warp.x, 2.0f * warp.y, warp.x)), 6));
    sf tone = fbm(vadds(vadd(vmul(q, 5.0f), off), 3.0f), 4);
    sv color = vmix(xyzs(body[kMaterial]), xyzs(body[kSurfaceColor]), dark * 0.85f);
    color = vmul(color, 0.85f + 0.3f * tone);
    sf streak = fbm(vadds(vadd(V(q.x * 4.0f, q.y * 4.0f, q.z * 18.0f), off), 9.0f), 3);
    color = vmul(color, 0.95f + 0.1f * streak);
    color = vmul(color, craters(q, sf(body[kSurfaceColor].w), off, 0.0f, 0.45f, 0.0f));
    sf ice = polar_caps(q, sf(body[kSurfaceParams].x), off);
    return vmix(color, V(0.92f, 0.92f, 0.94f), ice);
}

/* ice_plates: pathtrace.wgsl:691-708 */
static __device__ __noinline__ sv ice_plates(sv p) {
    sv base = vfloor(p);
    sf nearest = 10.0f, second = 10.0f, tone = 0.0f;
    for (int i = 0; i < 27; i++) {
        sv cell = vadd(base, V((float)(i % 3 - 1), (float)((i / 3) % 3 - 1), (float)(i / 9 - 1)));
        sv delta = vsub(vadd(vadds(cell, 0.2f), vmul(hash33(cell), 0.6f)), p);
        sf d = vdot(delta, delta);
        if (d < nearest) {
            second = nearest;
            nearest = d;
            tone = hash31(vadds(cell, 57.0f));
        } else {
            second = minf_(second, d);
        }
    }
    return V(sqrtf(nearest), sqrtf(second) - sqrtf(nearest), tone);
}

/* icy_albedo: pathtrace.wgsl:714-766 */
static __device__ __noinline__ sv icy_albedo(const float4 *body, sv q) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sv ice = xyzs(body[kMaterial]);
    sv rust = vmulv(xyzs(body[kSurfaceColor]), V(0.72f, 0.62f, 0.56f));
    sv b = vadd(vmul(q, 3.1f), off);
    sv warp = vsubs(V(fbm(vadds(b, 11.0f), 3), fbm(vadds(b, 23.0f), 3), fbm(vadds(b, 37.0f), 3)), 0.5f);
    sf terrain = fbm(vadd(vadd(vmul(q, 4.2f), off), warp), 5);
    sf rubble = fbm(vadd(vadd(vmul(q, 85.0f), off), vmul(warp, 7.0f)), 4);
    sf chaos = smoothstepf(0.42f, 0.65f, terrain + 0.14f * (rubble - 0.5f));
    sv plates = ice_plates(vadd(vadd(vmul(q, 72.0f), off), vmul(warp, 4.0f)));
    sf seams = 1.0f - smoothstepf(0.015f, 0.07f, plates.y);
    sf dust = chaos * (0.2f + 0.46f * rubble + 0.18f * plates.z);
    sv color = vmix(ice, rust, dust);
    color = vmix(color, vmul(rust, 0.8f), seams * chaos * 0.35f);
    sf ridged_plain = ridge(fbm(vadds(vadd(vmul(q, 34.0f), off), 83.0f), 3), 0.025f);
    color = vmix(color, rust, ridged_plain * (0.1f + 0.14f * chaos));
    color = vmul(color, 0.87f + 0.22f * fbm(vadd(vmul(q, 180.0f), off), 3));
    sv warped = vadd(q, vmul(warp, 0.1f));
    sf roughness = 0.0015f * (rubble - 0.5f);
    sf shoulder = 0.0f, fissure = 0.0f, fresh_ridge = 0.0f;
    for (uint32_t i = 0; i < 64u; i++) {
        sv h = hash33(vadd(off, V((float)i * 3.7f, 1.0f, 2.0f)));
        sv family = hash33(vadd(off, V((float)(i / 8u) * 17.3f, 21.0f, 7.0f)));
        sv n = vnormalize(vadd(vsubs(vmul(family, 2.0f), 1.0f), vmul(vsubs(vmul(h, 2.0f), 1.0f), 0.28f)));
        sf shift = (hash31(vadd(off, V((float)i, 9.0f, 4.0f))) - 0.5f) * 1.4f;
        sf width = (i < 10u ? 0.0015f + 0.0022f * h.z : 0.0005f + 0.0011f * h.z) *
                      (0.65f + 0.8f * vnoise(vadd(vmul(q, 17.0f), vmul(h, 29.0f))));
        sf bend = 0.03f * (vnoise(vadd(vmul(q, 6.0f), vmul(family, 31.0f))) - 0.5f) +
                     0.008f * (vnoise(vadd(vmul(q, 24.0f), vmul(family, 37.0f))) - 0.5f);
        sf dist = fabsf(vdot(warped, n) - shift + roughness + bend);
        sf along = smoothstepf(0.28f, 0.62f, vnoise(vadd(vmul(q, 3.5f), vmul(h, 50.0f))));
        shoulder = maxf_(shoulder, (1.0f - smoothstepf(width, width * 4.0f, dist)) * along);
        sf double_ridge = fabsf(dist - width * 0.85f);
        sf single = 1.0f - smoothstepf(width * 0.25f, width, dist);
        sf paired = 1.0f - smoothstepf(width * 0.15f, width * 0.55f, double_ridge);
        fissure = maxf_(fissure, (i < 10u ? paired : single) * along);
        fresh_ridge = maxf_(fresh_ridge,
                            (1.0f - smoothstepf(width * 0.15f, width * 0.35f, fabsf(dist - width * 1.8f))) * along);
    }
    color = vmix(color, rust, shoulder * 0.17f);
    color = vmix(color, vmul(rust, 0.7f), fissure * 0.8f);
    color = vmix(color, ice, fresh_ridge * 0.13f);
    return vmul(color, craters(q, sf(body[kSurfaceColor].w) * 0.2f, off, 0.0f, 0.3f, 0.4f));
}

/* volcanic_albedo: pathtrace.wgsl:770-850 */
static __device__ __noinline__ sv volcanic_albedo(const float4 *body, sv q) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sv sulphur = xyzs(body[kMaterial]), deposit = xyzs(body[kSurfaceColor]);
    sv b = vadd(vmul(q, 4.7f), off);
    sv warp = vsubs(V(fbm(b, 3), fbm(vadds(b, 19.0f), 3), fbm(vadds(b, 41.0f), 3)), 0.5f);
    sf terrain = fbm(vadd(vadd(vmul(q, 10.0f), off), vmul(warp, 2.0f)), 6);
    sf weathered = smoothstepf(0.38f, 0.65f, fbm(vadds(vadd(vmul(q, 3.7f), off), 11.0f), 5));
    sf fine = fbm(vadd(vadd(vmul(q, 90.0f), off), vmul(warp, 3.0f)), 4);
    sv crust = vmix(vmulv(sulphur, V(0.43f, 0.51f, 0.6f)), deposit, 0.12f);
    sv color = vmul(sulphur, 0.7f + 0.5f * terrain);
    color = vmix(color, crust, weathered * (0.45f + 0.5f * terrain));
    sf frost = smoothstepf(0.38f, 0.74f, fbm(vadd(vadds(vadd(vmul(q, 6.0f), off), 29.0f), warp), 5) + 0.2f * (fine - 0.5f));
    sv frost_color = vmix(sulphur, V(0.72f, 0.7f, 0.62f), 0.8f);
    color = vmix(color, frost_color, frost * 0.7f);
    sf flow_edges = ridge(fbm(vadd(vadd(vmul(q, 35.0f), off), vmul(warp, 2.0f)), 4), 0.025f);
    color = vmix(color, crust, flow_edges * weathered * 0.4f);
    color = vmul(color, (0.82f + 0.32f * fine) * (0.94f + 0.13f * fbm(vadd(vmul(q, 210.0f), off), 3)));
    sf dark = 0.0f, ash = 0.0f, red = 0.0f, white = 0.0f;
    sf density = sf(body[kSurfaceColor].w);
    sf scale = 5.5f;
    sv p = vadds(vadd(vmul(q, scale), off), 300.0f);
    sv base = vfloor(p);
    for (int i = 0; i < 27; i++) {
        sv cell = vadd(base, V((float)(i % 3 - 1), (float)((i / 3) % 3 - 1), (float)(i / 9 - 1)));
        if (hash31(vadd(cell, V(4.0f, 41.0f, 9.0f))) > 0.6f * density) continue;
        sv centre;
        if (!cell_centre(cell, cell, scale, vadds(off, 300.0f), &centre)) continue;
        sf size = hash31(vadd(cell, V(8.0f, 1.0f, 3.0f)));
        sf radius = (0.025f + 0.11f * size * size * size) / scale;
        sv offset = vsub(q, centre);
        sf reach = vlength(offset) * scale;
        if (reach > 0.95f) continue;
        sf cutoff = 1.0f - smoothstepf(0.75f, 0.95f, reach);
        sv tangent = vcross(centre, V(0.37f, 0.83f, 0.41f));
        sv east = vdivs(tangent, maxf_(vlength(tangent), 1.0e-5f));
        sv north = vcross(centre, east);
        sf angle = TAU_F * hash31(vadds(cell, 91.0f));
        sf ux = vdot(offset, east) / radius, uy = vdot(offset, north) / radius;
        sf ca = cos_d(angle), sa = sin_d(angle);
        sf uvx = ux * ca - uy * sa, uvy = ux * sa + uy * ca;
        sf ragged = fbm(vadd(V(uvx * 2.7f, uvy * 2.7f, 0.0f), vmul(cell, 7.0f)), 3) - 0.5f;
        sf sx = uvx * (1.0f / (0.65f + 0.9f * size)), sy = uvy * 1.0f;
        sf d = sqrtf(sx * sx + sy * sy) + 0.42f * ragged;
        sf pit = 1.0f - smoothstepf(0.68f, 0.86f, d);
        sf age = hash31(vadds(cell, 31.0f));
        sf fx = uvx - (0.2f + 2.3f * age), fy = uvy - 0.35f * sin_d(uvx * 1.3f + angle);
        sf gx = fx * (0.75f - 0.48f * age), gy = fy * (0.85f + 0.35f * size);
        sf flow_shape = sqrtf(gx * gx + gy * gy) + 0.65f * ragged +
                           0.35f * (fbm(vadd(V(uvx * 1.8f, uvy * 1.8f, 0.0f), vmul(cell, 3.0f)), 4) - 0.5f);
        sf flow = (1.0f - smoothstepf(0.72f, 0.9f, flow_shape)) * smoothstepf(0.35f, 0.85f, age) * 0.85f;
        dark = maxf_(dark, maxf_(pit, flow) * cutoff);
        sf plume = hash31(vadd(cell, V(2.0f, 6.0f, 17.0f)));
        sf hx = (uvx - 0.5f) * 0.16f, hy = (uvy - 0.3f) * 0.23f;
        sf halo = exp_d(-(hx * hx + hy * hy)) * cutoff;
        ash = maxf_(ash, halo * (0.25f + 0.35f * age));
        white = maxf_(white, halo * stepf(0.45f, plume) * (1.0f - stepf(0.83f, plume)));
        sf apron = surface_gaussian((sqrtf(uvx * uvx + uvy * uvy) + ragged - 3.5f) / 1.6f) *
                      (0.25f + 0.75f * smoothstepf(-1.5f, 2.0f, uvy));
        red = maxf_(red, apron * stepf(0.83f, plume) * cutoff);
    }
    color = vmix(color, vmul(crust, 0.7f), ash * 0.45f);
    color = vmix(color, frost_color, white * 0.4f);
    color = vmix(color, vmulv(deposit, V(0.85f, 0.7f, 0.65f)), red * 0.6f);
    return vmix(color, V(0.035f, 0.032f, 0.026f), dark * 0.96f);
}

/* terran_albedo: pathtrace.wgsl:854-895 */
static __device__ __noinline__ sv terran_albedo(const float4 *body, sv q) {
    sv off = seed_offset(sf(body[kAxisY].w));
    sv land_base = xyzs(body[kMaterial]), ocean = xyzs(body[kSurfaceColor]);
    sv b = vadd(vmul(q, 1.5f), off);
    sv warp = vsubs(V(fbm(b, 4), fbm(vadds(b, 13.0f), 4), fbm(vadds(b, 29.0f), 4)), 0.5f);
    sf height = fbm(vadd(vadd(vmul(q, 1.1f), off), vmul(warp, 0.9f)), 7);
    sf sea = 0.5f + (sf(body[kSurfaceParams].y) - 0.5f) * 0.3f;
    sf coast = smoothstepf(sea, sea + 0.004f, height);
    sf shallow = 1.0f - smoothstepf(sea - 0.04f, sea, height);
    sv water = vmix(vadd(vmul(ocean, 1.8f), V(0.0f, 0.04f, 0.05f)), ocean, shallow);
    sf moisture = fbm(vadds(vadd(vmul(q, 3.0f), off), 41.0f), 5) + 0.25f * (fabsf(q.z) - 0.35f);
    sv green = vmulv(land_base, V(0.45f, 0.62f, 0.38f));
    sv land = vmix(land_base, green, smoothstepf(0.45f, 0.6f, moisture));
    sf altitude = smoothstepf(sea + 0.08f, sea + 0.2f, height);
    land = vmix(land, V(0.42f, 0.38f, 0.34f), altitude * 0.6f);
    land = vmix(land, V(0.9f, 0.9f, 0.92f), smoothstepf(sea + 0.19f, sea + 0.24f, height));
    land = vmul(land, 0.88f + 0.24f * fbm(vadd(vmul(q, 25.0f), off), 3));
    sv color = vmix(water, land, coast);
    sf ice = polar_caps(q, sf(body[kSurfaceParams].x), off);
    color = vmix(color, V(0.9f, 0.92f, 0.95f), ice);
    sf cover = sf(body[kSurfaceParams].z);
    if (cover > 0.0f) {
        sv c1 = vadd(vmul(q, 1.6f), off);
        sv w1 = vsubs(V(fbm(vadds(c1, 77.0f), 4), fbm(vadds(c1, 91.0f), 4), 0.5f), 0.5f);
        sv c2 = vadd(vadd(vmul(q, 4.0f), off), vmul(w1, 3.0f));
        sv w2 = vsubs(V(fbm(c2, 4), fbm(vadd(vadds(vadd(vmul(q, 4.0f), off), 17.0f), vmul(w1, 3.0f)), 4), 0.5f), 0.5f);
        sv cq = vadd(vadd(vadd(V(q.x * 2.5f, q.y * 2.5f, q.z * 7.0f), off), vmul(w1, 2.5f)), vmul(w2, 1.2f));
        sf cloud = fbm(cq, 7);
        sf lat = fabsf(q.z);
        sf belts = 0.06f * (surface_gaussian(lat / 0.12f) + surface_gaussian((lat - 0.72f) / 0.15f)) -
                      0.04f * surface_gaussian((lat - 0.42f) / 0.1f);
        sf threshold = 0.62f - 0.22f * cover - belts;
        sf mask = smoothstepf(threshold - 0.04f, threshold + 0.14f, cloud);
        color = vmix(color, V(0.93f, 0.94f, 0.96f), mask * 0.95f);
    }
    return color;
}

/* surface_albedo, styles 1-6 (pathtrace.wgsl:897-910): clamped to [0, 1]. */
static __device__ __noinline__ sv style_albedo(const float4 *body, uint32_t style, sv local) {
    sv c;
    switch (style) {
        case 1u: c = gas_giant_albedo(body, local); break;
        case 2u: c = cratered_albedo(body, local); break;
        case 3u: c = rocky_albedo(body, local); break;
        case 4u: c = icy_albedo(body, local); break;
        case 5u: c = volcanic_albedo(body, local); break;
        default: c = terran_albedo(body, local); break;
    }
    return V(clampf_(c.x, 0.0f, 1.0f), clampf_(c.y, 0.0f, 1.0f), clampf_(c.z, 0.0f, 1.0f));
}


// terrain_shading (terrain.wgsl:142-150): on alpine ground a steep
// triangle shades with its own flat face.
__device__ __forceinline__ float3 alpine_face_shading(float3 smooth_normal, float3 a, float3 b, float3 c) {
    const sv pa = V(a.x, a.y, a.z), pb = V(b.x, b.y, b.z), pc = V(c.x, c.y, c.z);
    sv face = vnormalize(vcross(vsub(pb, pa), vsub(pc, pa)));
    if (face.y < sf(0.0f)) face = V(-face.x, -face.y, -face.z);
    const sv n = V(smooth_normal.x, smooth_normal.y, smooth_normal.z);
    return to_f3(vnormalize(vmix(n, face, smoothstepf(0.25f, 0.5f, sf(1.0f) - face.y))));
}

/* ---------------------------------------------------------------- */
/* Vegetation primitives (kinds 3 conifer, 4 grass, 5 trunk):        */
/* forest.wgsl:56-136, in the primitive's frame. (normal, distance), */
/* distance 1e30 on a miss. Strict f32, correctly rounded            */
/* transcendentals.                                                  */
/* ---------------------------------------------------------------- */
struct veg_hit {
    sv n;
    sf t;
};
// terrain_triangle (terrain.wgsl:102-116) in this arithmetic: (u, v, t).
__device__ __forceinline__ sv tri_hit(sv o, sv d, sv a, sv b, sv c) {
    const sv ab = vsub(b, a), ac = vsub(c, a);
    const sv p = vcross(d, ac);
    const sf determinant = vdot(ab, p);
    if (fabsf(determinant) < sf(1.0e-12f)) return V(0.0f, 0.0f, 1.0e30f);
    const sf inverse = sf(1.0f) / determinant;
    const sv relative = vsub(o, a);
    const sf u = vdot(relative, p) * inverse;
    const sv q = vcross(relative, ab);
    const sf v = vdot(d, q) * inverse;
    const sf distance = vdot(ac, q) * inverse;
    if (u < sf(-1.0e-6f) || v < sf(-1.0e-6f) || u + v > sf(1.000001f) || distance <= sf(0.001f))
        return V(0.0f, 0.0f, 1.0e30f);
    return V(u, v, distance);
}
__device__ __forceinline__ sv vneg(sv a) { return V(-a.x, -a.y, -a.z); }
static __device__ __noinline__ veg_hit trunk_hit(sv p, sv d, sv e) {
    sv o = V(p.x / e.x, p.y / e.y, p.z / e.z);
    sv v = V(d.x / e.x, d.y / e.y, d.z / e.z);
    veg_hit result{V(0.0f, 0.0f, 0.0f), sf(1.0e30f)};
    sf a = v.x * v.x + v.z * v.z;
    sf b = o.x * v.x + o.z * v.z;
    sf c = o.x * o.x + o.z * o.z - 1.0f;
    sf disc = b * b - a * c;
    if (a > 1.0e-15f && disc >= 0.0f) {
        for (uint32_t side = 0; side < 2u; side++) {
            sf t = (-b + (side == 1u ? sqrtf(disc) : -sqrtf(disc))) / a;
            sv q = vadd(o, vmul(v, t));
            if (t > 0.001f && t < result.t && fabsf(q.y) <= 1.0f) {
                result.n = vnormalize(V(q.x / e.x, 0.0f / e.y, q.z / e.z));
                result.t = t;
            }
        }
    }
    if (fabsf(v.y) > 1.0e-15f) {
        for (uint32_t side = 0; side < 2u; side++) {
            sf sign_y = side == 1u ? 1.0f : -1.0f;
            sf t = (sign_y - o.y) / v.y;
            sv q = vadd(o, vmul(v, t));
            if (t > 0.001f && t < result.t && q.x * q.x + q.z * q.z <= 1.0f) {
                result.n = V(0.0f, sign_y, 0.0f);
                result.t = t;
            }
        }
    }
    return result;
}
static __device__ __noinline__ veg_hit conifer_hit(sv p, sv d, sv e) {
    veg_hit result = trunk_hit(vadd(p, V(0.0f, e.y * 0.08f, 0.0f)), d, V(e.x * 0.065f, e.y * 0.92f, e.z * 0.065f));
    sv o = V(p.x / e.x, p.y / e.y, p.z / e.z);
    sv v = V(d.x / e.x, d.y / e.y, d.z / e.z);
    for (uint32_t tier = 0; tier < 6u; tier++) {
        sf t = (float)tier;
        sf base = -0.6f + t * 0.27f;
        sf height = minf_(0.66f - t * 0.045f, 1.0f - base);
        sf radius = 0.94f - t * 0.148f;
        sf ox = sin_d(t * 4.1f) * 0.022f, oz = cos_d(t * 3.7f) * 0.022f;
        sv q = vsub(o, V(ox, base + height, oz));
        sf k = radius / height;
        sf a = v.x * v.x + v.z * v.z - k * k * v.y * v.y;
        sf b = q.x * v.x + q.z * v.z - k * k * q.y * v.y;
        sf c = q.x * q.x + q.z * q.z - k * k * q.y * q.y;
        sf disc = b * b - a * c;
        if (fabsf(a) < 1.0e-12f || disc < 0.0f) continue;
        for (uint32_t side = 0; side < 2u; side++) {
            sf distance = (-b + (side == 1u ? sqrtf(disc) : -sqrtf(disc))) / a;
            sv h = vadd(q, vmul(v, distance));
            if (distance <= 0.001f || distance >= result.t || h.y > 0.0f || h.y < -height) continue;
            sf angle = atan2_d(h.z, h.x);
            sf skirt = -h.y / height;
            sf branches = 0.5f + 0.5f * sin_d(angle * (9.0f + t) + t * 3.7f);
            sf needle = vnoise(vadds(vmulv(vadd(p, vmul(d, distance)), V(9.0f, 17.0f, 9.0f)), t * 7.0f));
            if (skirt > 0.76f + 0.19f * branches || (skirt > 0.4f && needle < 0.26f)) continue;
            result.n = vnormalize(V(h.x / e.x, -k * k * h.y / e.y, h.z / e.z));
            result.t = distance;
        }
    }
    return result;
}
static __device__ __noinline__ veg_hit grass_hit(sv p, sv d, sv e) {
    veg_hit result{V(0.0f, 0.0f, 0.0f), sf(1.0e30f)};
    for (uint32_t blade = 0; blade < 9u; blade++) {
        sf i = (float)blade;
        sf angle = i * 2.39996f;
        sv side = V(cos_d(angle), 0.0f, sin_d(angle));
        sv base = vsub(vmul(vmul(side, e.x), 0.15f), V(0.0f, e.y, 0.0f));
        sv tip = vadd(vmul(vmul(side, e.x), 0.6f + 0.3f * sin_d(i * 3.0f)),
                      V(0.0f, e.y * (0.5f + 0.5f * cos_d(i * 1.3f)), 0.0f));
        sv width = vmul(V(-side.z, 0.0f, side.x), 0.035f);
        sv hit = tri_hit(p, d, vsub(base, width), vadd(base, width), tip);
        if (hit.z < result.t) {
            sv normal = vnormalize(vcross(width, vsub(tip, base)));
            if (vdot(normal, d) > 0.0f) normal = vneg(normal);
            result.n = normal;
            result.t = hit.z;
        }
    }
    return result;
}
/* The vegetation branch of landscape_query (ground.wgsl:197-202). */
static __device__ __noinline__ veg_hit vegetation_hit(sf kind, sv p, sv d, sv e) {
    if (kind < 3.5f) return conifer_hit(p, d, e);
    if (kind < 4.5f) return grass_hit(p, d, e);
    return trunk_hit(p, d, e);
}

}  // namespace style

// surface_albedo's styled branch (pathtrace.wgsl:897-910): the body's ten
// staged float4 words and the body-local normal.
static __device__ __noinline__ float3 styled_albedo(const float4 *body, uint32_t style_code, float3 local) {
    const style::sv c = style::style_albedo(body, style_code, style::V(local.x, local.y, local.z));
    return style::to_f3(c);
}

// surface_albedo (pathtrace.wgsl:897-925): a procedural style when
// axis_x.w rounds to 1-6, else the colour with the optional mottle.
// `Styled` compiles the styles in: the kernels of frames without styled
// bodies (or air) leave the call out, and with it its register cost.
template <bool Styled>
__device__ __forceinline__ float3 surface_albedo(const Scene &S, uint32_t i, float3 normal) {
    if constexpr (Styled) {
        const float4 axis_x = bf(S, i, kAxisX);
        if (axis_x.w >= 0.5f) {
            const float3 x = xyz(axis_x), y = xyz(bf(S, i, kAxisY));
            const float3 local = f3(dot_rn(normal, x), dot_rn(normal, y), dot_rn(normal, cross_rn(x, y)));
            return styled_albedo(S.B + i * kBodyVec4, (uint32_t)(axis_x.w + 0.5f), local);
        }
    }
    const float4 material = bf(S, i, kMaterial);
    const float strength = bf(S, i, kLow).w;
    const float m = strength > 0.0f ? mottle(xyz(bf(S, i, kAxisX)), bf(S, i, kAxisY), strength, normal) : 1.0f;
    return f3(clampf(material.x * m, 0.0f, 1.0f), clampf(material.y * m, 0.0f, 1.0f),
              clampf(material.z * m, 0.0f, 1.0f));
}

}  // namespace sg
