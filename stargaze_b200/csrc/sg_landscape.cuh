// sg_landscape.cuh — metre-scale local landscape for the B200 integrator.
//
// Follows src/shaders/ground.wgsl (host sphere in the surface frame, props
// with group-marker bounds, materials, 5 mm bounce offset) and
// src/shaders/terrain.wgsl (min/max quadtree over a triangulated
// heightfield, geometry cache). Everything that decides a hit — the
// surface-frame origin, the host quadratic, slab and facet tests, the
// quadtree intervals and Moller-Trumbore triangles — uses explicit
// round-to-nearest operations so hit ids and distances match an IEEE f32
// evaluation of the WGSL bit for bit. Materials and bump normals use FMA.
//
// Extensions over the reference (stated where they apply): the traversal
// stack holds 40 entries so 4096-cell grids (34 entries deep) fit; prop
// lists may exceed 256 entries (nested group markers form a BVH); an
// optional scalar albedo map replaces the theme floor.
#pragma once

#include "sg_device.cuh"

namespace sg {

constexpr float kMetresPerAu = 149597870700.0f;
constexpr uint32_t kLocalBase = SG_LOCAL_BASE;
constexpr uint32_t kTerrainId = SG_TERRAIN_ID;
constexpr int kTerrainStack = 40;

__device__ __forceinline__ float3 g_east(const Scene &S) { return f3(S.s->g.ground_east[0], S.s->g.ground_east[1], S.s->g.ground_east[2]); }
__device__ __forceinline__ float3 g_up(const Scene &S) { return f3(S.s->g.ground_up[0], S.s->g.ground_up[1], S.s->g.ground_up[2]); }
__device__ __forceinline__ float3 g_north(const Scene &S) { return f3(S.s->g.ground_north[0], S.s->g.ground_north[1], S.s->g.ground_north[2]); }

// to_ground / from_ground / camera_origin / ground_origin (ground.wgsl:17-32).
__device__ __forceinline__ float3 to_ground(const Scene &S, float3 v) {
    return f3(dot_rn(v, g_east(S)), dot_rn(v, g_up(S)), dot_rn(v, g_north(S)));
}
__device__ __forceinline__ float3 from_ground(const Scene &S, float3 v) {
    return add_rn(add_rn(mul_rn(g_east(S), v.x), mul_rn(g_up(S), v.y)), mul_rn(g_north(S), v.z));
}
__device__ __forceinline__ float3 camera_origin(const Scene &S, const Ray &r) {
    if (r.anchor == kMiss) return r.o;
    return add_rn(xyz(bf(S, r.anchor, kCenter)), add_rn(xyz(bf(S, r.anchor, kLow)), r.o));
}
__device__ __forceinline__ float3 ground_origin(const Scene &S, const Ray &r) {
    const float3 g = to_ground(S, mul_rn(camera_origin(S, r), kMetresPerAu));
    return f3(g.x, __fadd_rn(g.y, S.s->g.ground_east[3]), g.z);
}

// The same in double for the FP64 sites (metres per AU exact).
constexpr double kMetresPerAuD = 149597870700.0;
__device__ __forceinline__ d3 to_ground_d(const Scene &S, d3 v) {
    return d3{dot(v, D(g_east(S))), dot(v, D(g_up(S))), dot(v, D(g_north(S)))};
}
__device__ __forceinline__ d3 from_ground_d(const Scene &S, d3 v) {
    return D(g_east(S)) * v.x + D(g_up(S)) * v.y + D(g_north(S)) * v.z;
}
__device__ __forceinline__ d3 ground_origin_d(const Scene &S, const Ray &r) {
    d3 c = D(r.o);
    if (r.anchor != kMiss) c = D(xyz(bf(S, r.anchor, kCenter))) + D(xyz(bf(S, r.anchor, kLow))) + c;
    d3 g = to_ground_d(S, c * kMetresPerAuD);
    g.y += (double)S.s->g.ground_east[3];
    return g;
}

// rotate_north / rotate_east / rotate_up and the tumbled-rock frame
// (ground.wgsl:33-61). Sines and cosines come precomputed per primitive
// (TraceParams::prop_trig: (sin, cos) of the x, y and z angles, the yaw in
// the z slot), evaluated in double on the host and rounded to f32.
__device__ __forceinline__ float3 rotate_north(float3 p, float s, float c) {
    return f3(__fsub_rn(__fmul_rn(c, p.x), __fmul_rn(s, p.y)), __fadd_rn(__fmul_rn(s, p.x), __fmul_rn(c, p.y)), p.z);
}
__device__ __forceinline__ float3 rotate_east(float3 p, float s, float c) {
    return f3(p.x, __fsub_rn(__fmul_rn(c, p.y), __fmul_rn(s, p.z)), __fadd_rn(__fmul_rn(s, p.y), __fmul_rn(c, p.z)));
}
__device__ __forceinline__ float3 rotate_up(float3 p, float s, float c) {
    return f3(__fadd_rn(__fmul_rn(c, p.x), __fmul_rn(s, p.z)), p.y, __fadd_rn(__fmul_rn(-s, p.x), __fmul_rn(c, p.z)));
}
// t0 = (sin x, cos x, sin y, cos y), t1 = (sin z, cos z, -, -).
__device__ __forceinline__ float3 rock_to_local(float3 p, float4 t0, float4 t1) {
    return rotate_east(rotate_up(rotate_north(p, -t1.x, t1.y), -t0.z, t0.w), -t0.x, t0.y);
}
__device__ __forceinline__ float3 rock_from_local(float3 p, float4 t0, float4 t1) {
    return rotate_north(rotate_up(rotate_east(p, t0.x, t0.y), t0.z, t0.w), t1.x, t1.y);
}

__device__ __forceinline__ float comp(float3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
__device__ __forceinline__ float3 div3_rn(float3 a, float3 b) {
    return f3(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y), __fdiv_rn(a.z, b.z));
}

// box_interval (ground.wgsl:64-78): slabs with explicit parallel handling.
__device__ __forceinline__ float2 box_interval(float3 p, float3 d, float3 extent) {
    float n = -1.0e30f, f = 1.0e30f;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        const float pa = comp(p, axis), da = comp(d, axis), ea = comp(extent, axis);
        if (fabsf(da) < 1.0e-12f) {
            if (fabsf(pa) > ea) return make_float2(1.0e30f, -1.0e30f);
        } else {
            const float a = __fdiv_rn(__fsub_rn(-ea, pa), da);
            const float b = __fdiv_rn(__fsub_rn(ea, pa), da);
            n = fmaxf(n, fminf(a, b));
            f = fminf(f, fmaxf(a, b));
        }
    }
    return make_float2(n, f);
}

// rock_hit (ground.wgsl:82-121): a box with clipped corners; 14 planes.
static __device__ __noinline__ float4 rock_hit(float3 p, float3 d, float3 e) {
    const float3 origin = div3_rn(p, e);
    const float3 direction = div3_rn(d, e);
    float near_ = -1.0e30f, far_ = 1.0e30f;
    float3 near_normal = f3(0.0f, 0.0f, 0.0f), far_normal = f3(0.0f, 0.0f, 0.0f);
#pragma unroll 1
    for (uint32_t face = 0; face < 14u; ++face) {
        float3 n = f3(0.0f, 0.0f, 0.0f);
        float limit = 1.0f;
        if (face < 6u) {
            const float s = (face & 1u) == 1u ? 1.0f : -1.0f;
            const uint32_t axis = face / 2u;
            n = f3(axis == 0u ? s : 0.0f, axis == 1u ? s : 0.0f, axis == 2u ? s : 0.0f);
        } else {
            const uint32_t bits = face - 6u;
            n = f3((bits & 1u) ? 1.0f : -1.0f, (bits & 2u) ? 1.0f : -1.0f, (bits & 4u) ? 1.0f : -1.0f);
            limit = __fadd_rn(1.65f, __fmul_rn(0.08f, (float)(bits % 3u)));
        }
        const float denominator = dot_rn(n, direction);
        const float gap = __fsub_rn(limit, dot_rn(n, origin));
        if (fabsf(denominator) < 1.0e-12f) {
            if (gap < 0.0f) return make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
        } else {
            const float distance = __fdiv_rn(gap, denominator);
            if (denominator < 0.0f && distance > near_) {
                near_ = distance;
                near_normal = div3_rn(n, e);
            }
            if (denominator > 0.0f && distance < far_) {
                far_ = distance;
                far_normal = div3_rn(n, e);
            }
        }
        if (near_ > far_) return make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
    }
    if (far_ <= 0.001f) return make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
    const float3 nn = near_ > 0.001f ? normalize(near_normal) : normalize(far_normal);
    return make_float4(nn.x, nn.y, nn.z, near_ > 0.001f ? near_ : far_);
}

// ---------------------------------------------------------------------------
// Heightfield (terrain.wgsl)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t t_cells(const sg_settings *s) {
    const uint32_t log2 = s->g.ground_counts[2] >> 8;
    return log2 != 0u ? (1u << log2) : 512u;
}
__host__ __device__ __forceinline__ uint32_t t_width(uint32_t cells) { return cells + 1u; }
__host__ __device__ __forceinline__ uint32_t t_vertices(uint32_t cells) { return t_width(cells) * t_width(cells); }
__host__ __device__ __forceinline__ bool t_compact(uint32_t cells) { return cells > 1024u; }
__host__ __device__ __forceinline__ uint32_t t_vertex_stride(uint32_t cells) { return t_compact(cells) ? 2u : 6u; }
__host__ __device__ __forceinline__ uint32_t t_nodes(uint32_t cells) {
    const uint32_t leaves = cells / 2u;
    return (4u * leaves * leaves - 1u) / 3u;
}
__host__ __device__ __forceinline__ uint32_t t_bounds(uint32_t cells) {
    return (t_compact(cells) ? 1u : 3u) * t_vertices(cells);
}
__host__ __device__ __forceinline__ uint32_t t_cache(uint32_t cells) { return t_bounds(cells) + 2u * t_nodes(cells); }
__host__ __device__ __forceinline__ uint32_t t_vertex_cache(uint32_t cells) { return t_cache(cells) + 6u * t_nodes(cells); }

__device__ __forceinline__ float t_scale_r(float r) { return clampf(__fdiv_rn(r, 200000.0f), 0.0001f, 1.0f); }
__device__ __forceinline__ float t_coordinate(uint32_t i, uint32_t cells, float scale) {
    const float u = __fsub_rn(__fdiv_rn(__fmul_rn(2.0f, (float)i), (float)cells), 1.0f);
    return __fmul_rn(__fmul_rn(__fmul_rn(u, fabsf(u)), 16000.0f), scale);
}
__device__ __forceinline__ float t_curvature(float px, float pz, float r) {
    const float d2 = __fadd_rn(__fmul_rn(px, px), __fmul_rn(pz, pz));
    return __fdiv_rn(-d2, __fadd_rn(r, __fsqrt_rn(fmaxf(__fsub_rn(__fmul_rn(r, r), d2), 0.0f))));
}
__host__ __device__ __forceinline__ uint32_t compact_bits(uint32_t value) {
    uint32_t x = value & 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0f0f0f0fu;
    x = (x | (x >> 4)) & 0x00ff00ffu;
    return (x | (x >> 8)) & 0x0000ffffu;
}
// Heap index -> (x, z, size) (terrain.wgsl:169-173).
__device__ __forceinline__ uint3 t_node(uint32_t index, uint32_t cells) {
    const uint32_t level = (31u - __clz(3u * index + 1u)) / 2u;
    const uint32_t size = cells >> level;
    const uint32_t morton = index - ((1u << (2u * level)) - 1u) / 3u;
    return make_uint3(compact_bits(morton) * size, compact_bits(morton >> 1) * size, size);
}

__device__ __forceinline__ float3 t_vertex(const float *T, uint32_t cells, float scale, uint32_t x, uint32_t z) {
    const float *v = T + t_vertex_cache(cells) + (size_t)(z * t_width(cells) + x) * t_vertex_stride(cells);
    if (t_compact(cells)) return f3(t_coordinate(x, cells, scale), v[0], t_coordinate(z, cells, scale));
    return f3(v[0], v[1], v[2]);
}
__device__ __forceinline__ float3 t_normal(const float *T, uint32_t cells, uint32_t x, uint32_t z) {
    const float *v = T + t_vertex_cache(cells) + (size_t)(z * t_width(cells) + x) * t_vertex_stride(cells);
    if (t_compact(cells)) {
        const uint32_t packed = (uint32_t)v[1];
        const float xx = __fsub_rn(__fmul_rn(__fdiv_rn((float)(packed & 4095u), 4095.0f), 2.0f), 1.0f);
        const float zz = __fsub_rn(__fmul_rn(__fdiv_rn((float)(packed >> 12), 4095.0f), 2.0f), 1.0f);
        const float y = __fsqrt_rn(fmaxf(__fsub_rn(1.0f, __fadd_rn(__fmul_rn(xx, xx), __fmul_rn(zz, zz))), 1.0e-6f));
        const float3 n = f3(xx, y, zz);
        return mul_rn(n, __fdiv_rn(1.0f, length_rn(n)));
    }
    return f3(v[3], v[4], v[5]);
}

// terrain_triangle (terrain.wgsl:65-81): (u, v, distance).
__device__ __forceinline__ float3 t_triangle(float3 o, float3 d, float3 a, float3 b, float3 c) {
    const float3 ab = sub_rn(b, a), ac = sub_rn(c, a);
    const float3 p = cross_rn(d, ac);
    const float determinant = dot_rn(ab, p);
    if (fabsf(determinant) < 1.0e-12f) return f3(0.0f, 0.0f, 1.0e30f);
    const float inverse = __fdiv_rn(1.0f, determinant);
    const float3 relative = sub_rn(o, a);
    const float u = __fmul_rn(dot_rn(relative, p), inverse);
    const float3 q = cross_rn(relative, ab);
    const float v = __fmul_rn(dot_rn(d, q), inverse);
    const float distance = __fmul_rn(dot_rn(ac, q), inverse);
    if (u < -1.0e-6f || v < -1.0e-6f || __fadd_rn(u, v) > 1.000001f || distance <= 0.001f)
        return f3(0.0f, 0.0f, 1.0e30f);
    return f3(u, v, distance);
}

// terrain_interval (terrain.wgsl:118-130).
__device__ __forceinline__ float2 t_interval(const float *T, uint32_t cells, float3 o, float3 inv, uint32_t index) {
    const float *c = T + t_cache(cells) + (size_t)index * 6u;
    const float3 lo = f3(c[0], c[1], c[2]), hi = f3(c[3], c[4], c[5]);
    const bool px = fabsf(inv.x) >= 1.0e29f, py = fabsf(inv.y) >= 1.0e29f, pz = fabsf(inv.z) >= 1.0e29f;
    if ((px && (o.x < lo.x || o.x > hi.x)) || (py && (o.y < lo.y || o.y > hi.y)) || (pz && (o.z < lo.z || o.z > hi.z)))
        return make_float2(1.0e30f, -1.0e30f);
    const float ax = __fmul_rn(__fsub_rn(lo.x, o.x), inv.x), bx = __fmul_rn(__fsub_rn(hi.x, o.x), inv.x);
    const float ay = __fmul_rn(__fsub_rn(lo.y, o.y), inv.y), by = __fmul_rn(__fsub_rn(hi.y, o.y), inv.y);
    const float az = __fmul_rn(__fsub_rn(lo.z, o.z), inv.z), bz = __fmul_rn(__fsub_rn(hi.z, o.z), inv.z);
    const float ex = px ? -1.0e30f : fminf(ax, bx), ey = py ? -1.0e30f : fminf(ay, by), ez = pz ? -1.0e30f : fminf(az, bz);
    const float xx = px ? 1.0e30f : fmaxf(ax, bx), xy = py ? 1.0e30f : fmaxf(ay, by), xz = pz ? 1.0e30f : fmaxf(az, bz);
    return make_float2(fmaxf(ex, fmaxf(ey, ez)), fminf(xx, fminf(xy, xz)));
}

// terrain_query (terrain.wgsl:152-234): near-to-far min/max quadtree.
// Returns (normal, distance); distance 1e30 on a miss.
static __device__ __noinline__ float4 terrain_query(const float *T, uint32_t cells, float radius, float3 o, float3 d,
                                             float initial_limit, bool occlusion) {
    float4 result = make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
    float limit = initial_limit;
    const float scale = t_scale_r(radius);
    const float3 inv = f3(__fdiv_rn(d.x >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.x), 1.0e-30f)),
                          __fdiv_rn(d.y >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.y), 1.0e-30f)),
                          __fdiv_rn(d.z >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.z), 1.0e-30f)));
    const float2 root = t_interval(T, cells, o, inv, 0u);
    if (root.x > root.y || root.y <= 0.001f || root.x >= limit) return result;
    uint32_t stack_node[kTerrainStack];
    float stack_t[kTerrainStack];
    stack_node[0] = 0u;
    stack_t[0] = fmaxf(root.x, 0.0f);
    uint32_t count = 1u;
    while (count > 0u) {
        count -= 1u;
        if (stack_t[count] >= limit) continue;
        const uint32_t index = stack_node[count];
        const uint3 node = t_node(index, cells);
        if (node.z == 2u) {
#pragma unroll 1
            for (uint32_t z = node.y; z < node.y + 2u; ++z) {
#pragma unroll 1
                for (uint32_t x = node.x; x < node.x + 2u; ++x) {
                    const float3 a = t_vertex(T, cells, scale, x, z);
                    const float3 b = t_vertex(T, cells, scale, x + 1u, z);
                    const float3 c = t_vertex(T, cells, scale, x, z + 1u);
                    const float3 e = t_vertex(T, cells, scale, x + 1u, z + 1u);
                    const float3 first = t_triangle(o, d, a, c, b);
                    const float3 second = t_triangle(o, d, e, b, c);
                    if (first.z < limit) {
                        if (occlusion) return make_float4(0.0f, 0.0f, 0.0f, first.z);
                        const float3 n = normalize(t_normal(T, cells, x, z) * (1.0f - first.x - first.y) +
                                                   t_normal(T, cells, x, z + 1u) * first.x +
                                                   t_normal(T, cells, x + 1u, z) * first.y);
                        result = make_float4(n.x, n.y, n.z, first.z);
                        limit = first.z;
                    }
                    if (second.z < limit) {
                        if (occlusion) return make_float4(0.0f, 0.0f, 0.0f, second.z);
                        const float3 n = normalize(t_normal(T, cells, x + 1u, z + 1u) * (1.0f - second.x - second.y) +
                                                   t_normal(T, cells, x + 1u, z) * second.x +
                                                   t_normal(T, cells, x, z + 1u) * second.y);
                        result = make_float4(n.x, n.y, n.z, second.z);
                        limit = second.z;
                    }
                }
            }
        } else {
            uint32_t children[4];
            float distances[4];
#pragma unroll
            for (uint32_t child = 0; child < 4u; ++child) {
                children[child] = index * 4u + child + 1u;
                const float2 bounds = t_interval(T, cells, o, inv, children[child]);
                distances[child] =
                    (bounds.x <= bounds.y && bounds.y > 0.001f && bounds.x < limit) ? fmaxf(bounds.x, 0.0f) : 1.0e30f;
            }
            // Far first on the stack: the nearest child is popped first.
#pragma unroll
            for (uint32_t i = 1; i < 4u; ++i) {
#pragma unroll
                for (uint32_t j = i; j > 0u; --j) {
                    if (distances[j - 1u] >= distances[j]) break;
                    const float dd = distances[j - 1u];
                    const uint32_t cc = children[j - 1u];
                    distances[j - 1u] = distances[j];
                    children[j - 1u] = children[j];
                    distances[j] = dd;
                    children[j] = cc;
                }
            }
#pragma unroll
            for (uint32_t i = 0; i < 4u; ++i) {
                if (distances[i] < limit && count < (uint32_t)kTerrainStack) {
                    stack_node[count] = children[i];
                    stack_t[count] = distances[i];
                    count += 1u;
                }
            }
        }
    }
    return result;
}

// landscape_top (ground.wgsl:244-251).
__device__ __forceinline__ float landscape_top(const Scene &S) {
    float top = __uint_as_float(S.s->g.ground_counts[3]);
    if (S.s->g.ground_counts[1] != 0u && S.p->terrain) top = fmaxf(top, S.p->terrain[t_cache(S.p->terrain_cells) + 4u]);
    return top;
}

// The host-sphere intersection of landscape_query (ground.wgsl:138-158) in
// double; the returned distance (AU) and normal are rounded to f32.
static __device__ __noinline__ LandHit host_sphere_fp64(Scene S, Ray ray, float limit, bool occlusion) {
    const LandHit miss{limit, kMiss, 0.0f, f3(0.0f, 0.0f, 0.0f)};
    const double radius = (double)S.s->g.ground_up[3];
    const d3 o = ground_origin_d(S, ray);
    const d3 d = to_ground_d(S, D(ray.d));
    const double a = dot(d, d);
    const double b = -radius * d.y - dot(o, d);
    const double c = o.x * o.x + o.z * o.z + o.y * (2.0 * radius + o.y);
    const double h = b * b - a * c;
    if (h < 0.0) return miss;
    const double root = sqrt(h);
    const double q = b + (b >= 0.0 ? root : -root);
    if (q == 0.0) return miss;
    const double cq = c / q, qa = q / a;
    const double t0 = fmin(cq, qa), t1 = fmax(cq, qa);
    const double distance = t0 > 0.001 ? t0 : t1;
    const float au = (float)(distance / kMetresPerAuD);
    if (!(distance > 0.001) || !(au < limit)) return miss;
    if (occlusion) return LandHit{au, kLocalBase, 0.0f, f3(0.0f, 0.0f, 0.0f)};
    const d3 p = o + d * distance;
    d3 n = d3{p.x / radius, 1.0 + p.y / radius, p.z / radius};
    n = n * (1.0 / sqrt(dot(n, n)));
    return LandHit{au, kLocalBase, 0.0f, F(from_ground_d(S, n))};
}

// landscape_query (ground.wgsl:123-242). Vegetation kinds (> 2.5) are
// rejected on the host and never reach the device.
template <bool C, bool L, bool F>
static __device__ SG_HELPER LandHit landscape_query(Scene S, Counter<C, L, F> K, Ray ray, float limit, bool occlusion) {
    LandHit closest{limit, kMiss, 0.0f, f3(0.0f, 0.0f, 0.0f)};
    const sg_settings *s = S.s;
    if (s->g.ground_north[3] == 0.0f) return closest;
    const float3 o = ground_origin(S, ray);
    const float3 d = to_ground(S, ray.d);
    const float radius = s->g.ground_up[3];
    if (dot_rn(o, o) > __fmul_rn(__fmul_rn(4.0f, radius), radius)) {
        // Distant paths keep the celestial cross-product intersection.
        const uint32_t host = (uint32_t)s->g.ground_north[3] - 1u;
        float delta;
        const float t = sphere_distance(S, K, ray, host, b_radius(S, host), delta);
        if (t >= 1.0e30f) return LandHit{1.0e30f, kMiss, 0.0f, f3(0.0f, 0.0f, 0.0f)};
        return LandHit{t, host, delta, sphere_normal(S, ray, host, delta)};
    }
    if (d.y >= 0.0f && o.y > landscape_top(S)) return closest;
    if constexpr (F) {
        const LandHit host = host_sphere_fp64(S, ray, closest.t, occlusion);
        if (host.index != kMiss) {
            if (occlusion) return host;
            closest = host;
        }
    } else {
    // Host sphere in the surface frame (ground.wgsl:138-158).
    const float a = dot_rn(d, d);
    const float b = __fsub_rn(__fmul_rn(-radius, d.y), dot_rn(o, d));
    const float c = __fadd_rn(__fadd_rn(__fmul_rn(o.x, o.x), __fmul_rn(o.z, o.z)),
                              __fmul_rn(o.y, __fadd_rn(__fmul_rn(2.0f, radius), o.y)));
    const float h = __fsub_rn(__fmul_rn(b, b), __fmul_rn(a, c));
    if (h >= 0.0f) {
        const float root = __fsqrt_rn(h);
        const float q = __fadd_rn(b, b >= 0.0f ? root : -root);
        if (q != 0.0f) {
            const float cq = __fdiv_rn(c, q), qa = __fdiv_rn(q, a);
            const float t0 = fminf(cq, qa), t1 = fmaxf(cq, qa);
            const float distance = t0 > 0.001f ? t0 : t1;
            const float au = __fdiv_rn(distance, kMetresPerAu);
            if (distance > 0.001f && au < closest.t) {
                if (occlusion) return LandHit{au, kLocalBase, 0.0f, f3(0.0f, 0.0f, 0.0f)};
                const float3 p = add_rn(o, mul_rn(d, distance));
                const float3 n = normalize(f3(p.x / radius, 1.0f + p.y / radius, p.z / radius));
                closest = LandHit{au, kLocalBase, 0.0f, from_ground(S, n)};
            }
        }
    }
    }
    if (s->g.ground_counts[1] != 0u && S.p->terrain) {
        const float tl = __fmul_rn(fminf(closest.t, 1.0e18f), kMetresPerAu);
        const float4 terrain = terrain_query(S.p->terrain, S.p->terrain_cells, radius, o, d, tl, occlusion);
        if (terrain.w < tl && terrain.w < 1.0e29f) {
            closest = LandHit{__fdiv_rn(terrain.w, kMetresPerAu), kTerrainId, 0.0f, from_ground(S, xyz(terrain))};
            if (occlusion) return closest;
        }
    }
    const uint32_t n_objects = s->g.ground_counts[0];
    const float4 *objects = S.p->props;
#pragma unroll 1
    for (uint32_t i = 0; i < n_objects; ++i) {
        const float4 oc = objects[3u * i];
        const float4 oe = objects[3u * i + 1u];
        const float3 center = xyz(oc), e = xyz(oe);
        const float kind = oc.w;
        if (kind < 0.0f) {
            // Group marker: skip the subtree when its bounds are missed.
            const float2 bounds = box_interval(sub_rn(o, center), d, e);
            if (bounds.x > bounds.y || bounds.y <= 0.001f || __fdiv_rn(bounds.x, kMetresPerAu) > closest.t)
                i += (uint32_t)(-kind);
            continue;
        }
        float3 p = sub_rn(o, center), v = d;
        const float4 t0 = S.p->prop_trig[2u * i], t1 = S.p->prop_trig[2u * i + 1u];
        if (kind == 2.25f) {
            p = rock_to_local(p, t0, t1);
            v = rock_to_local(v, t0, t1);
        } else {
            p = rotate_north(p, -t1.x, t1.y);
            v = rotate_north(v, -t1.x, t1.y);
        }
        float distance = 1.0e30f;
        float3 n = f3(0.0f, 0.0f, 0.0f);
        if (kind > 1.5f) {
            const float2 bounds = box_interval(p, v, e);
            if (bounds.x > bounds.y || bounds.y <= 0.001f || __fdiv_rn(bounds.x, kMetresPerAu) > closest.t) continue;
            const float4 rock = rock_hit(p, v, e);
            distance = rock.w;
            n = xyz(rock);
        } else if (kind > 0.5f) {
            const float3 sp = div3_rn(p, e), sd = div3_rn(v, e);
            const float aa = dot_rn(sd, sd), bb = dot_rn(sp, sd), cc = __fsub_rn(dot_rn(sp, sp), 1.0f);
            const float hh = __fsub_rn(__fmul_rn(bb, bb), __fmul_rn(aa, cc));
            if (hh >= 0.0f) {
                const float root = __fsqrt_rn(hh);
                distance = __fdiv_rn(__fsub_rn(-bb, root), aa);
                if (distance <= 0.001f) distance = __fdiv_rn(__fadd_rn(-bb, root), aa);
                const float3 hp = add_rn(p, mul_rn(v, distance));
                n = normalize(f3(hp.x / (e.x * e.x), hp.y / (e.y * e.y), hp.z / (e.z * e.z)));
            }
        } else {
            const float2 interval = box_interval(p, v, e);
            if (interval.x <= interval.y && interval.y > 0.001f) {
                distance = interval.x > 0.001f ? interval.x : interval.y;
                const float3 point = div3_rn(add_rn(p, mul_rn(v, distance)), e);
                const float3 ap = f3(fabsf(point.x), fabsf(point.y), fabsf(point.z));
                const float sx = point.x > 0.0f ? 1.0f : (point.x < 0.0f ? -1.0f : 0.0f);
                const float sy = point.y > 0.0f ? 1.0f : (point.y < 0.0f ? -1.0f : 0.0f);
                const float sz = point.z > 0.0f ? 1.0f : (point.z < 0.0f ? -1.0f : 0.0f);
                if (ap.x >= ap.y && ap.x >= ap.z) n.x = sx;
                else if (ap.y >= ap.z) n.y = sy;
                else n.z = sz;
            }
        }
        const float au = __fdiv_rn(distance, kMetresPerAu);
        if (distance > 0.001f && distance < 1.0e29f && au < closest.t) {
            if (occlusion) return LandHit{au, kLocalBase + 1u + i, 0.0f, f3(0.0f, 0.0f, 0.0f)};
            n = kind == 2.25f ? rock_from_local(n, t0, t1) : rotate_north(n, t1.x, t1.y);
            closest = LandHit{au, kLocalBase + 1u + i, 0.0f, from_ground(S, n)};
        }
    }
    return closest;
}

// ---------------------------------------------------------------------------
// Local shading (ground.wgsl:252-317, :597-662)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 landscape_point(const Scene &S, const Ray &ray, float t) {
    return add_rn(ground_origin(S, ray), mul_rn(to_ground(S, ray.d), __fmul_rn(t, kMetresPerAu)));
}
__device__ __forceinline__ float3 mix3(float3 a, float3 b, float t) {
    return f3(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t));
}
__device__ __forceinline__ float footprint_of(const sg_settings *s, float distance) {
    return distance * 2.0f * s->g.cam_forward[3] / fmaxf(s->g.viewport[1], 1.0f);
}

static __device__ __noinline__ float3 forest_floor(float3 p, float footprint, float3 normal) {
    const float broad = vnoise(add_rn(mul_rn(p, 0.045f), f3(7.0f, 0.0f, 13.0f)));
    const float middle = vnoise(p * 0.7f);
    const float grain = vnoise(p * 18.0f);
    const float detail = 1.0f - smoothstepf(0.006f, 0.055f, footprint);
    const float3 moss = mix3(f3(0.028f, 0.054f, 0.014f), f3(0.105f, 0.14f, 0.039f), middle);
    const float3 earth = mix3(f3(0.055f, 0.029f, 0.013f), f3(0.17f, 0.115f, 0.057f), middle);
    float3 color = mix3(earth, moss, smoothstepf(0.35f, 0.63f, broad));
    const float needles = powf(fmaxf(0.0f, sinf(p.x * 92.0f + p.z * 137.0f + middle * 7.0f)), 18.0f) *
                          smoothstepf(0.50f, 0.68f, grain);
    color = mix3(color, f3(0.22f, 0.145f, 0.067f), needles * detail * 0.5f);
    color = color * (1.0f + (grain - 0.5f) * 0.38f * detail);
    const float slope = 1.0f - fmaxf(normal.y, 0.0f);
    const float3 stone = mix3(f3(0.095f, 0.105f, 0.10f), f3(0.24f, 0.23f, 0.20f), middle);
    color = mix3(color, stone, smoothstepf(0.10f, 0.43f, slope + (broad - 0.5f) * 0.17f));
    const float center = 2.0f + 0.30f * p.z + 2.0f * sinf(p.z * 0.055f);
    const float edge = fabsf(p.x - center) + (middle - 0.5f) * 0.55f;
    const float path = (1.0f - smoothstepf(0.8f, 2.1f, edge)) * (1.0f - smoothstepf(45.0f, 95.0f, p.z)) *
                       smoothstepf(-10.0f, 0.0f, p.z);
    const float3 gravel =
        mix3(f3(0.12f, 0.095f, 0.062f), f3(0.26f, 0.23f, 0.17f), grain * detail + 0.5f * (1.0f - detail));
    return mix3(color, gravel, path * 0.85f);
}
static __device__ __noinline__ float3 desert_floor(float3 p, float footprint, float3 normal) {
    const float broad = vnoise(add_rn(mul_rn(p, 0.007f), f3(19.0f, 2.0f, 4.0f)));
    const float gravel = vnoise(p * 2.8f);
    const float detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    const float3 sand = mix3(f3(0.31f, 0.21f, 0.125f), f3(0.53f, 0.40f, 0.26f), broad);
    const float3 rock = mix3(f3(0.18f, 0.10f, 0.055f), f3(0.38f, 0.245f, 0.145f), broad);
    float3 color = mix3(sand, rock, smoothstepf(0.08f, 0.4f, 1.0f - fmaxf(normal.y, 0.0f)));
    color = color * (1.0f + (gravel - 0.5f) * 0.32f * detail);
    const float center = 2.8f + 0.55f * sinf(p.z / 38.0f) + 1.4f * sinf(p.z / 210.0f);
    const float edge = fabsf(p.x - center);
    const float aa = fmaxf(0.015f, footprint * 0.5f);
    const float fade = (1.0f - smoothstepf(0.25f, 0.9f, footprint)) *
                       (1.0f - smoothstepf(1000.0f, 2200.0f, fabsf(p.z))) *
                       (1.0f - smoothstepf(0.12f, 0.35f, 1.0f - fmaxf(normal.y, 0.0f)));
    const float worn = 1.0f - smoothstepf(0.8f, 1.2f, edge);
    const float rut_edge = fabsf(edge - 0.68f) + (gravel - 0.5f) * 0.1f * detail;
    const float tracks = 1.0f - smoothstepf(0.12f - aa, 0.23f + aa, rut_edge);
    const float3 packed = sand * (0.72f + 0.10f * gravel * detail);
    color = mix3(color, sand * 0.93f, worn * fade * 0.35f);
    return mix3(color, packed, tracks * fade * 0.8f);
}
static __device__ __noinline__ float3 crater_floor(float3 p, float footprint, float3 normal) {
    const float broad = vnoise(add_rn(mul_rn(p, 0.004f), f3(3.0f, 0.0f, 8.0f)));
    const float middle = vnoise(p * 0.09f);
    const float grain = vnoise(p * 3.1f);
    const float detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    float tone = mixf(0.11f, 0.21f, broad) * (0.86f + 0.28f * middle);
    tone *= 1.0f + 0.35f * smoothstepf(0.15f, 0.5f, 1.0f - fmaxf(normal.y, 0.0f));
    tone *= 1.0f + (grain - 0.5f) * 0.3f * detail;
    return f3(tone, tone * 0.97f, tone * 0.93f);
}

// Albedo-map extension: index of the nearest texel at surface-frame (x, z).
__device__ __forceinline__ uint32_t map_texel(const TraceParams *P, float3 p) {
    const float u = (p.x / P->map_extent + 1.0f) * 0.5f * (float)P->map_width;
    const float w = (p.z / P->map_extent + 1.0f) * 0.5f * (float)P->map_height;
    int i = (int)floorf(u), j = (int)floorf(w);
    i = max(0, min(i, (int)P->map_width - 1));
    j = max(0, min(j, (int)P->map_height - 1));
    return (uint32_t)j * P->map_width + (uint32_t)i;
}

// landscape_albedo (ground.wgsl:597-632), themes 0-2, plus the map.
static __device__ __noinline__ float3 landscape_albedo(Scene S, Ray ray, float t, uint32_t index, float3 normal) {
    const float3 p = landscape_point(S, ray, t);
    const float distance = t * kMetresPerAu;
    const float3 n = to_ground(S, normal);
    if (index == kLocalBase || index == kTerrainId) {
        if (S.p->albedo_map) {
            const float a = S.p->albedo_map[map_texel(S.p, p)];
            return f3(a, a, a);
        }
        const float footprint = footprint_of(S.s, distance);
        const uint32_t theme = S.s->g.ground_counts[2] & 255u;
        if (theme == 1u) return desert_floor(p, footprint, n);
        if (theme == 2u) return crater_floor(p, footprint, n);
        return forest_floor(p, footprint, n);
    }
    const float4 albedo = S.p->props[3u * (index - kLocalBase - 1u) + 2u];
    const float3 tint = xyz(albedo);
    const float kind = albedo.w;
    if (kind == 0.0f) return tint;
    const float middle = vnoise(p * 1.7f);
    const float fine = mixf(vnoise(p * 12.0f), 0.5f, smoothstepf(18.0f, 110.0f, distance));
    if (kind > 4.5f) return tint * (0.65f + 0.6f * middle);
    const float strata = sinf(p.y * 8.0f + 2.5f * middle);
    const float lichen = smoothstepf(0.52f, 0.76f, middle) * fmaxf(n.y, 0.0f);
    const float3 stone = tint * (0.7f + 0.45f * fine + 0.07f * strata);
    if ((S.s->g.ground_counts[2] & 255u) != 0u) return stone;
    return mix3(stone, f3(0.11f, 0.145f, 0.037f), lichen * 0.65f);
}

// landscape_shading_normal (ground.wgsl:633-648), themes 0-2.
static __device__ __noinline__ float3 landscape_shading_normal(Scene S, Ray ray, float t, uint32_t index, float3 normal) {
    if (index != kLocalBase && index != kTerrainId) return normal;
    const float3 p = landscape_point(S, ray, t);
    const float distance = t * kMetresPerAu;
    const float strength = 0.11f * (1.0f - smoothstepf(8.0f, 65.0f, distance));
    const float dx = vnoise((p + f3(0.025f, 0.0f, 0.0f)) * 6.0f) - vnoise((p - f3(0.025f, 0.0f, 0.0f)) * 6.0f);
    const float dz = vnoise((p + f3(0.0f, 0.0f, 0.025f)) * 6.0f) - vnoise((p - f3(0.0f, 0.0f, 0.025f)) * 6.0f);
    const float3 g = g_east(S) * (-dx) + g_north(S) * (-dz);
    return normalize(normal + g * strength);
}

// landscape_outgoing in double (FP64 sites): the hit point, its reprojection
// onto the host sphere and the 5 mm step, rounded to f32 AU at the end.
static __device__ __noinline__ Ray landscape_outgoing_fp64(Scene S, Ray ray, float t, uint32_t index, float3 normal) {
    d3 p = ground_origin_d(S, ray) + to_ground_d(S, D(ray.d)) * ((double)t * kMetresPerAuD);
    if (index == kLocalBase) {
        const double radius = (double)S.s->g.ground_up[3];
        const double d2 = p.x * p.x + p.z * p.z;
        if (p.y > -radius && d2 < radius * radius) p.y = -d2 / (radius + sqrt(radius * radius - d2));
    }
    p = p + to_ground_d(S, D(normal)) * 0.005;
    p.y -= (double)S.s->g.ground_east[3];
    return Ray{F(from_ground_d(S, p) * (1.0 / kMetresPerAuD)), normal, kMiss};
}

// landscape_outgoing (ground.wgsl:649-662): reproject a host-sphere hit
// without radius cancellation, step 5 mm along the normal, back to AU.
template <bool F>
__device__ __forceinline__ Ray landscape_outgoing(const Scene &S, const Ray &ray, float t, uint32_t index,
                                                  float3 normal) {
    if constexpr (F) return landscape_outgoing_fp64(S, ray, t, index, normal);
    float3 p = landscape_point(S, ray, t);
    if (index == kLocalBase) {
        const float radius = S.s->g.ground_up[3];
        const float d2 = __fadd_rn(__fmul_rn(p.x, p.x), __fmul_rn(p.z, p.z));
        if (p.y > -radius && d2 < __fmul_rn(radius, radius))
            p.y = __fdiv_rn(-d2, __fadd_rn(radius, __fsqrt_rn(__fsub_rn(__fmul_rn(radius, radius), d2))));
    }
    p = add_rn(p, mul_rn(to_ground(S, normal), 0.005f));
    p.y = __fsub_rn(p.y, S.s->g.ground_east[3]);
    return Ray{div_rn(from_ground(S, p), kMetresPerAu), normal, kMiss};
}

}  // namespace sg
