// sg_air.cuh — the host planet's air: single-scattering Rayleigh + Mie
// along the camera ray with planetshine (pathtrace.wgsl:927-1234), the
// extinction of light and continuations that cross it, and the surface sky
// cache that lights local ground (terrain.wgsl:286-339).
//
// The reference runs the camera ray's air as its own pass per sample
// (integrate_camera_air, pathtrace.wgsl:1629-1643) and hands trace() the
// in-scatter and the random state after it; trace() then re-derives the
// view transmittance (camera_air_transmittance, :1217-1234). Here the
// integrator calls atmosphere() in place at the camera ray's first vertex:
// its random state there is the one the separate pass starts from (the
// same camera draws and point-disc draw), and its t_view is the product
// camera_air_transmittance recomputes, so one call yields both.
//
// Everything here is out of line: it runs only in frames with air, and
// keeps the airless stages' register allocation.
#pragma once

#include "sg_device.cuh"
#include "sg_landscape.cuh"

namespace sg {

namespace {

constexpr uint32_t kAtmoViewSteps = 8u;  // ATMO_VIEW_STEPS (pathtrace.wgsl:67)
constexpr uint32_t kAtmoSunSteps = 4u;   // ATMO_SUN_STEPS (pathtrace.wgsl:68)
constexpr uint32_t kSkyTexels = 128u;    // 16 azimuths x 8 elevations

__device__ __forceinline__ float3 atmo_center(const Scene &S) {
    return f3(S.s->g.atmo_center[0], S.s->g.atmo_center[1], S.s->g.atmo_center[2]);
}
__device__ __forceinline__ float host_radius(const Scene &S) { return S.s->g.atmo_center[3]; }
__device__ __forceinline__ float atmosphere_top(const Scene &S) {
    return S.s->g.atmo_center[3] + S.s->g.atmo_params[2];
}
__device__ __forceinline__ float atmo_scale_height(const Scene &S) { return S.s->g.atmo_params[1]; }
__device__ __forceinline__ float3 beta_extinction(const Scene &S) {
    const float *r = S.s->g.atmo_rayleigh;
    return f3(r[0] + r[3], r[1] + r[3], r[2] + r[3]);
}
__device__ __forceinline__ float3 exp_neg(float3 beta, float x) {
    return f3(expf(-beta.x * x), expf(-beta.y * x), expf(-beta.z * x));
}
// u32(ceil(x)) clamped to [2, ATMO_VIEW_STEPS]; the conversion saturates.
__device__ __forceinline__ uint32_t view_steps(float x) {
    const float q = ceilf(x);
    if (!(q > 2.0f)) return 2u;
    if (q >= (float)kAtmoViewSteps) return kAtmoViewSteps;
    return (uint32_t)q;
}

// shell_exit (pathtrace.wgsl:945-956): distance to the top of the air along
// `dir`, 0 when the ray never reaches the shell.
__device__ __forceinline__ float shell_exit(const Scene &S, float3 origin, float3 dir) {
    const float3 oc = origin - atmo_center(S);
    const float b = dot(oc, dir);
    const float top = atmosphere_top(S);
    const float c = dot(oc, oc) - top * top;
    const float disc = b * b - c;
    if (disc < 0.0f) return 0.0f;
    return -b + sqrtf(disc);
}

// density_integral (pathtrace.wgsl:959-974): midpoint column of exp(-h/H).
__device__ __forceinline__ float density_integral(const Scene &S, float3 origin, float3 dir, uint32_t steps) {
    const float distance = shell_exit(S, origin, dir);
    if (distance <= 0.0f) return 0.0f;
    const float dt = distance / (float)steps;
    const float inv_h = 1.0f / atmo_scale_height(S);
    const float r = host_radius(S);
    const float3 c = atmo_center(S);
    float sum = 0.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < steps; ++i) {
        const float3 p = origin + dir * (((float)i + 0.5f) * dt);
        const float h = fmaxf(length(p - c) - r, 0.0f);
        sum += expf(-h * inv_h);
    }
    return sum * dt;
}

// host_offset, inside_air (pathtrace.wgsl:976-992).
__device__ __forceinline__ float3 host_offset(const Scene &S, const Ray &origin) {
    if (origin.anchor == kMiss) return origin.o - atmo_center(S);
    return ((xyz(bf(S, origin.anchor, kCenter)) - atmo_center(S)) + xyz(bf(S, origin.anchor, kLow))) + origin.o;
}
__device__ __forceinline__ bool inside_air(const Scene &S, const Ray &origin) {
    if (S.s->g.atmo_params[3] < 0.5f) return false;
    const float3 oc = host_offset(S, origin);
    const float top = atmosphere_top(S);
    return dot(oc, oc) < top * top;
}

// air_transmittance (pathtrace.wgsl:995-1002): extinction from a point in
// the air to its top; points outside see none.
static __device__ __noinline__ float3 air_transmittance(Scene S, Ray origin, float3 dir) {
    if (!inside_air(S, origin)) return f3(1.0f, 1.0f, 1.0f);
    const float3 p = atmo_center(S) + host_offset(S, origin);
    return exp_neg(beta_extinction(S), density_integral(S, p, dir, kAtmoSunSteps));
}

// rayleigh_phase, mie_phase (pathtrace.wgsl:1004-1010), weighted by the
// scattering coefficients.
__device__ __forceinline__ float3 phase_weight(const Scene &S, float cos_theta) {
    const float *r = S.s->g.atmo_rayleigh;
    const float g = S.s->g.atmo_params[0];
    const float rayleigh = 3.0f / (16.0f * kPi) * (1.0f + cos_theta * cos_theta);
    const float g2 = g * g;
    const float mie = (1.0f - g2) / (4.0f * kPi * powf(1.0f + g2 - 2.0f * g * cos_theta, 1.5f));
    const float m = r[3] * mie;
    return f3(r[0] * rayleigh + m, r[1] * rayleigh + m, r[2] * rayleigh + m);
}

// sample_light_stratum (pathtrace.wgsl:214-230): one of `count` (1 or 4)
// equal-area strata of the light's cone.
template <bool C, bool L, bool F>
__device__ __forceinline__ LightSample sample_light_stratum(const Scene &S, Counter<C, L, F> K, const Ray &r,
                                                            uint32_t i, uint32_t stratum, uint32_t count,
                                                            uint32_t rng) {
    K.add(&Events::light_samples);
    const float3 oc = relative_center(S, r, i);
    const float3 axis = normalize(oc);
    const float width = cone_width_oc(oc, b_radius(S, i));
    float radial = rnd(K, rng);
    float azimuth = rnd(K, rng);
    if (count == 4u) {
        radial = ((float)(stratum & 1u) + radial) * 0.5f;
        azimuth = ((float)(stratum >> 1u) + azimuth) * 0.5f;
    }
    const float one_minus_cos = radial * width;
    const float sin_theta = sqrtf(one_minus_cos * (2.0f - one_minus_cos));
    float sp, cp;
    sincos_turn(azimuth, &sp, &cp);
    LightSample ls;
    ls.d = basis_direction(axis, sin_theta * cp, sin_theta * sp, 1.0f - one_minus_cos);
    ls.pdf = 1.0f / (kTau * width);
    ls.rng = rng;
    return ls;
}

// eclipse_light_samples (pathtrace.wgsl:239-262): four strata on a fresh
// accumulation (`counts_y`, the samples before this one, is 0) where a
// spherical limb may cross the light's disc, else one.
__device__ __forceinline__ uint32_t eclipse_light_samples(const Scene &S, const Ray &ray, uint32_t index,
                                                          uint32_t counts_y) {
    if (counts_y != 0u) return 1u;
    const float3 source = relative_center(S, ray, index);
    const float distance = length(source);
    const float3 axis = source / distance;
    const float source_chord = sqrtf(2.0f * cone_width_oc(source, b_radius(S, index)));
    const uint32_t n = S.s->counts[0];
#pragma unroll 1
    for (uint32_t b = 0; b < n; ++b) {
        if (b == index) continue;
        const float3 offset = relative_center(S, ray, b);
        const float d2 = dot(offset, offset);
        const float radius = b_radius(S, b);
        if (d2 <= radius * radius) continue;
        const float d = sqrtf(d2);
        if (d - radius >= distance + b_radius(S, index)) continue;
        const float sin2 = clampf(radius * radius / d2, 0.0f, 1.0f);
        const float limb_chord = sqrtf(2.0f * sin2 / (1.0f + sqrtf(1.0f - sin2)));
        const float separation = length(axis - offset / d);
        if (separation < source_chord + limb_chord && separation + source_chord > limb_chord) return 4u;
    }
    return 1u;
}

// air_light_visibility (rings.wgsl:121-141): above every landscape
// feature only bodies (the host included) and rings can shadow an air
// sample; among the landscape, the full surface test.
template <bool C, bool L, bool F>
__device__ __forceinline__ float air_light_visibility(const Scene &S, Counter<C, L, F> K, const Ray &ray,
                                                      uint32_t light) {
    if (S.s->g.ground_north[3] == 0.0f || ground_origin(S, ray).y <= landscape_top(S))
        return light_visibility(S, K, ray, light);
    float delta;
    const float surface = sphere_distance(S, K, ray, light, b_radius(S, light), delta);
    if (surface >= 1.0e30f) return 0.0f;
    const uint32_t n = S.s->counts[0];
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (i == light) continue;
        const float t = sphere_distance(S, K, ray, i, b_radius(S, i), delta);
        if (t < 1.0e30f && (t < surface || (t == surface && i < light))) return 0.0f;
    }
    float transmission = 1.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const RingHit h = ring_hit(S, K, ray, i);
        if (h.index != kMiss && h.t < surface) transmission *= ring_transmission(S, ray, h);
    }
    return transmission;
}

// sample_reflector (pathtrace.wgsl:1017-1044): one non-emissive body other
// than the host, by apparent solid angle x brightest albedo channel.
struct Reflector {
    uint32_t index;
    float inverse_probability;
};
template <bool C, bool L, bool F>
__device__ __forceinline__ Reflector sample_reflector(const Scene &S, Counter<C, L, F> K, float3 origin,
                                                      uint32_t &rng) {
    const Ray ray{origin, f3(0.0f, 0.0f, -1.0f), kMiss};
    const uint32_t host = (uint32_t)S.s->g.atmo_params[3] - 1u;
    uint32_t selected = kMiss;
    float selected_weight = 0.0f, total = 0.0f;
    const uint32_t n = S.s->counts[0];
#pragma unroll 1
    for (uint32_t b = 0; b < n; ++b) {
        const float4 material = bf(S, b, kMaterial);
        if (b == host || material.w > 0.5f) continue;
        const float weight =
            cone_width_oc(relative_center(S, ray, b), b_radius(S, b)) * fmaxf(material.x, fmaxf(material.y, material.z));
        if (weight <= 0.0f) continue;
        total += weight;
        if (rnd(K, rng) * total < weight) {
            selected = b;
            selected_weight = weight;
        }
    }
    return Reflector{selected, total / fmaxf(selected_weight, 1.0e-30f)};
}

// reflected_radiance (pathtrace.wgsl:1049-1073): starlight reflected once
// at the sampled point of the reflector.
template <bool C, bool L, bool F>
__device__ __forceinline__ float3 reflected_radiance(const Scene &S, Counter<C, L, F> K, const Ray &ray,
                                                     uint32_t index, uint32_t &rng) {
    float delta;
    const float radius = b_radius(S, index);
    if (sphere_distance(S, K, ray, index, radius, delta) >= 1.0e30f) return f3(0.0f, 0.0f, 0.0f);
    const float3 normal = sphere_normal(S, ray, index, delta);
    const float3 albedo = surface_albedo<true>(S, index, normal);
    Ray outgoing{normal * (radius * (1.0f + 2.0e-6f)), normal, index};
    float3 radiance = f3(0.0f, 0.0f, 0.0f);
    const uint32_t n_lights = light_count(S.s);
#pragma unroll 1
    for (uint32_t slot = 0; slot < n_lights; ++slot) {
        const uint32_t s = light_index(S.s, slot);
        const float4 material = bf(S, s, kMaterial);
        if (material.w < 0.5f) continue;
        const LightSample light = sample_light(S, K, outgoing, s, rng);
        rng = light.rng;
        const float cosine = fmaxf(dot(normal, light.d), 0.0f);
        if (cosine > 0.0f) {
            outgoing.d = light.d;
            radiance = radiance + albedo * xyz(material) *
                                      (cosine * light_visibility(S, K, outgoing, s) / (kPi * light.pdf));
        }
    }
    return radiance;
}

// ground_reflector_pdf (src/guided_ground.rs:21-37): the reflector half of
// the guided mixture's density along `ray` — every candidate's cone density
// where the ray hits it, weighted by its selection probability.
template <bool C, bool L, bool F>
static __device__ __noinline__ float ground_reflector_pdf(Scene S, Counter<C, L, F> K, Ray ray) {
    const uint32_t host = (uint32_t)S.s->g.atmo_params[3] - 1u;
    float total = 0.0f, density = 0.0f;
    const uint32_t n = S.s->counts[0];
#pragma unroll 1
    for (uint32_t b = 0; b < n; ++b) {
        const float4 material = bf(S, b, kMaterial);
        if (b == host || material.w > 0.5f) continue;
        const float radius = b_radius(S, b);
        const float width = cone_width_oc(relative_center(S, ray, b), radius);
        const float weight = width * fmaxf(material.x, fmaxf(material.y, material.z));
        if (weight <= 0.0f) continue;
        total += weight;
        float delta;
        if (sphere_distance(S, K, ray, b, radius, delta) < 1.0e30f) density += weight / (kTau * width);
    }
    return density / fmaxf(total, 1.0e-30f);
}

// brightest_risen_light (pathtrace.wgsl:1078-1089).
__device__ __forceinline__ float brightest_risen_light(const Scene &S, float3 origin) {
    const Ray ray{origin, f3(0.0f, 0.0f, -1.0f), kMiss};
    const float3 up = f3(S.s->g.ground_up[0], S.s->g.ground_up[1], S.s->g.ground_up[2]);
    float brightest = 0.0f;
    const uint32_t n_lights = light_count(S.s);
#pragma unroll 1
    for (uint32_t slot = 0; slot < n_lights; ++slot) {
        const uint32_t b = light_index(S.s, slot);
        const float4 material = bf(S, b, kMaterial);
        if (material.w < 0.5f) continue;
        const float3 oc = relative_center(S, ray, b);
        if (dot(normalize(oc), up) <= 0.0f) continue;
        brightest = fmaxf(brightest, fmaxf(material.x, fmaxf(material.y, material.z)) * kTau *
                                         cone_width_oc(oc, b_radius(S, b)));
    }
    return brightest;
}

// What atmosphere() leaves: view transmittance, in-scatter and the random
// state after its light samples.
struct AirScatter {
    float3 transmittance;
    float3 inscatter;
    uint32_t rng;
};

// atmosphere (pathtrace.wgsl:1092-1213): single scattering along a ray up
// to `limit` or the top of the air. `counts_y` is the sample's counts.y
// (the samples accumulated before it).
template <bool C, bool L, bool F>
static __device__ __noinline__ AirScatter atmosphere(Scene S, Counter<C, L, F> K, float3 origin, float3 dir,
                                                     float limit, uint32_t rng, uint32_t counts_y) {
    AirScatter result{f3(1.0f, 1.0f, 1.0f), f3(0.0f, 0.0f, 0.0f), rng};
    if (S.s->g.atmo_params[3] < 0.5f) return result;
    const float exit = shell_exit(S, origin, dir);
    const float t_max = fminf(limit, exit);
    if (t_max <= 0.0f) return result;
    const float3 beta_ext = beta_extinction(S);
    const float r = host_radius(S);
    const float scale_height = atmo_scale_height(S);
    const float3 center = atmo_center(S);
    const uint32_t steps = view_steps(t_max / (0.25f * scale_height));
    const float dt = t_max / (float)steps;
    // The WGSL select() evaluates the draw in every case; it changes nothing
    // but the separate jitter state.
    uint32_t jitter_rng = hash_u32(rng ^ 0x3c6ef372u);
    const float jittered = rnd(K, jitter_rng);
    const float jitter = (steps < kAtmoViewSteps || limit < exit) ? jittered : 0.5f;

    // Planetshine: one point of one reflector per camera ray, reused along
    // the column; its own random stream.
    uint32_t reflected_rng = hash_u32(rng ^ 0xa511e9b3u);
    const Reflector reflector = sample_reflector(S, K, origin, reflected_rng);
    float3 reflected = f3(0.0f, 0.0f, 0.0f), reflected_direction = dir, reflected_phase = f3(0.0f, 0.0f, 0.0f);
    if (reflector.index != kMiss) {
        Ray reflected_ray{origin, dir, kMiss};
        const LightSample light = sample_light(S, K, reflected_ray, reflector.index, reflected_rng);
        reflected_rng = light.rng;
        reflected_ray.d = light.d;
        reflected = reflected_radiance(S, K, reflected_ray, reflector.index, reflected_rng) *
                    (reflector.inverse_probability / light.pdf);
        reflected_direction = light.d;
        reflected_phase = phase_weight(S, dot(dir, light.d));
    }
    if (reflected.x > 0.0f || reflected.y > 0.0f || reflected.z > 0.0f) {
        const float sun = brightest_risen_light(S, origin);
        if (sun > 0.0f) {
            const float ratio = max3(reflected) / sun;
            const float minimum = 1.0f / sqrtf(clampf((float)counts_y + 1.0f, 1.0f, 4096.0f));
            const float keep = clampf(ratio * 1.0e3f, minimum, 1.0f);
            reflected = rnd(K, reflected_rng) < keep ? reflected / keep : f3(0.0f, 0.0f, 0.0f);
        }
    }
    const bool planetshine = reflected.x > 0.0f || reflected.y > 0.0f || reflected.z > 0.0f;

    const uint32_t n_lights = light_count(S.s);
    float3 t_view = f3(1.0f, 1.0f, 1.0f), inscatter = f3(0.0f, 0.0f, 0.0f);
#pragma unroll 1
    for (uint32_t i = 0; i < steps; ++i) {
        const float3 p = origin + dir * (((float)i + jitter) * dt);
        const float altitude = fmaxf(length(p - center) - r, 0.0f);
        const float column = expf(-altitude / scale_height) * dt;
        const float3 tau = beta_ext * column;
        const float3 step_t = f3(expf(-tau.x), expf(-tau.y), expf(-tau.z));
        // View extinction integrated over the segment; its thin limit.
        const float3 segment =
            f3(tau.x < 1.0e-3f ? column * (1.0f - 0.5f * tau.x) : (1.0f - step_t.x) / fmaxf(beta_ext.x, 1.0e-20f),
               tau.y < 1.0e-3f ? column * (1.0f - 0.5f * tau.y) : (1.0f - step_t.y) / fmaxf(beta_ext.y, 1.0e-20f),
               tau.z < 1.0e-3f ? column * (1.0f - 0.5f * tau.z) : (1.0f - step_t.z) / fmaxf(beta_ext.z, 1.0e-20f));
#pragma unroll 1
        for (uint32_t slot = 0; slot < n_lights; ++slot) {
            const uint32_t b = light_index(S.s, slot);
            const float4 material = bf(S, b, kMaterial);
            if (material.w < 0.5f) continue;
            Ray light_ray{p, dir, kMiss};
            const uint32_t light_samples = eclipse_light_samples(S, light_ray, b, counts_y);
#pragma unroll 1
            for (uint32_t k = 0; k < light_samples; ++k) {
                const LightSample light = sample_light_stratum(S, K, light_ray, b, k, light_samples, rng);
                rng = light.rng;
                light_ray.d = light.d;
                const float visibility = air_light_visibility(S, K, light_ray, b);
                if (visibility == 0.0f) continue;
                const float3 e_sun = xyz(material) * (visibility / ((float)light_samples * light.pdf));
                const float3 sun_t = exp_neg(beta_ext, density_integral(S, p, light.d, kAtmoSunSteps));
                const float3 beta_phase = phase_weight(S, dot(dir, light.d));
                inscatter = inscatter + t_view * segment * beta_phase * e_sun * sun_t;
            }
        }
        if (planetshine) {
            const float visibility = air_light_visibility(S, K, Ray{p, reflected_direction, kMiss}, reflector.index);
            if (visibility > 0.0f) {
                const float3 light_t = exp_neg(beta_ext, density_integral(S, p, reflected_direction, kAtmoSunSteps));
                inscatter = inscatter + t_view * segment * reflected_phase * reflected * (light_t * visibility);
            }
        }
        t_view = t_view * step_t;
    }
    result.transmittance = t_view;
    result.inscatter = inscatter;
    result.rng = rng;
    return result;
}

// surface_sky_lookup (terrain.wgsl:303-315): bilinear in the 16 x 8 cache
// over azimuth and the sine of elevation; zero below the horizon.
__device__ __forceinline__ float3 sky_texel(const float4 *sky, int x, int y) {
    const float4 t = sky[(uint32_t)min(max(y, 0), 7) * 16u + (uint32_t)((x + 16) % 16)];
    return f3(t.x, t.y, t.z);
}
static __device__ __noinline__ float3 surface_sky_lookup(Scene S, float3 dir) {
    const float4 *sky = S.p->sky_light;
    const float3 p = to_ground(S, dir);
    if (!sky || p.y <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float ux = fmodf(atan2f(p.z, p.x) / kTau + 1.0f, 1.0f) * 16.0f - 0.5f;
    const float uy = p.y * 8.0f - 0.5f;
    const float fx = floorf(ux), fy = floorf(uy);
    const int cx = (int)fx, cy = (int)fy;
    const float wx = ux - fx, wy = uy - fy;
    const float3 a0 = sky_texel(sky, cx, cy), a1 = sky_texel(sky, cx + 1, cy);
    const float3 b0 = sky_texel(sky, cx, cy + 1), b1 = sky_texel(sky, cx + 1, cy + 1);
    const float3 a = f3(mixf(a0.x, a1.x, wx), mixf(a0.y, a1.y, wx), mixf(a0.z, a1.z, wx));
    const float3 b = f3(mixf(b0.x, b1.x, wx), mixf(b0.y, b1.y, wx), mixf(b0.z, b1.z, wx));
    return f3(mixf(a.x, b.x, wy), mixf(a.y, b.y, wy), mixf(a.z, b.z, wy));
}

// surface_sky (terrain.wgsl:317-339): one cosine-distributed sky sample of
// a local surface at the depth limit, blocked by any opaque hit and
// attenuated by ring crossings.
struct SkySample {
    float3 radiance;
    uint32_t rng;
};
template <bool C, bool L, bool F>
static __device__ __noinline__ SkySample surface_sky(Scene S, Counter<C, L, F> K, Ray origin, float3 normal,
                                                     uint32_t rng) {
    const float u = rnd(K, rng);
    float sp, cp;
    sincos_turn(rnd(K, rng), &sp, &cp);
    const float su = sqrtf(u);
    const float3 dir = basis_direction(normal, su * cp, su * sp, sqrtf(1.0f - u));
    const float3 light = surface_sky_lookup(S, dir);
    if (max3(light) <= 0.0f) return SkySample{f3(0.0f, 0.0f, 0.0f), rng};
    const Ray ray{origin.o, dir, origin.anchor};
    const uint32_t n = S.s->counts[0];
    const float host = S.s->g.ground_north[3];
    // sky_blocked: any sphere but the landscape host, then the landscape.
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (host == (float)(i + 1u)) continue;
        float delta;
        if (sphere_distance(S, K, ray, i, b_radius(S, i), delta) < 1.0e30f) return SkySample{f3(0.0f, 0.0f, 0.0f), rng};
    }
    if constexpr (L) {
        if (landscape_query(S, K, ray, 1.0e30f, true).index != kMiss) return SkySample{f3(0.0f, 0.0f, 0.0f), rng};
    }
    float transmission = 1.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const RingHit h = ring_hit(S, K, ray, i);
        if (h.index != kMiss) transmission *= ring_transmission(S, ray, h);
    }
    return SkySample{light * transmission, rng};
}

}  // namespace

}  // namespace sg
