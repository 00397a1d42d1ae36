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
// The uploaded source: vertex bounds (heights, or heights and gradients)
// and each node's height range.
__host__ __device__ __forceinline__ uint32_t t_source(uint32_t cells) { return t_bounds(cells) + 2u * t_nodes(cells); }
// The node boxes (6 floats each) start 2 floats past a 16-byte boundary, so
// the four children of any node (indices 4k+1 .. 4k+4, 96 contiguous
// bytes) start on one: a node expansion reads them as six float4.
__host__ __device__ __forceinline__ uint32_t t_cache(uint32_t cells) {
    const uint32_t s = t_source(cells);
    return s + ((2u - (s & 3u)) & 3u);
}
__host__ __device__ __forceinline__ uint32_t t_vertex_cache(uint32_t cells) { return t_cache(cells) + 6u * t_nodes(cells); }

__device__ __forceinline__ float t_scale_r(float r) { return clampf(__fdiv_rn(r, 200000.0f), 0.0001f, 1.0f); }
// 2 i / cells: cells is a power of two, so the IEEE quotient is the exact
// product with 2^-log2(cells).
__device__ __forceinline__ float t_coordinate(uint32_t i, uint32_t cells, float scale) {
    const float inv_cells = __uint_as_float((127u - (31u - __clz(cells))) << 23);
    const float u = __fsub_rn(__fmul_rn(__fmul_rn(2.0f, (float)i), inv_cells), 1.0f);
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

// The cached (curved) height of a vertex of a compact grid.
__device__ __forceinline__ float t_height(const float *T, uint32_t cells, uint32_t x, uint32_t z) {
    return T[t_vertex_cache(cells) + (size_t)(z * t_width(cells) + x) * t_vertex_stride(cells)];
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

// terrain_interval (terrain.wgsl:118-130) of the box [lo, hi].
__device__ __forceinline__ float2 t_interval(float3 lo, float3 hi, float3 o, float3 inv) {
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
// With C, `ev` counts the interior nodes expanded and the triangles tested.
template <bool C>
static __device__ __noinline__ float4 terrain_query(const float *T, uint32_t cells, float radius, bool alpine, float3 o,
                                                    float3 d, float initial_limit, bool occlusion, Events *ev) {
    float4 result = make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
    float limit = initial_limit;
    const float scale = t_scale_r(radius);
    const float3 inv = f3(__fdiv_rn(d.x >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.x), 1.0e-30f)),
                          __fdiv_rn(d.y >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.y), 1.0e-30f)),
                          __fdiv_rn(d.z >= 0.0f ? 1.0f : -1.0f, fmaxf(fabsf(d.z), 1.0e-30f)));
    const float *rc = T + t_cache(cells);
    const float2 root = t_interval(f3(rc[0], rc[1], rc[2]), f3(rc[3], rc[4], rc[5]), o, inv);
    if (root.x > root.y || root.y <= 0.001f || root.x >= limit) return result;
    // Entries (node, entry distance bits): one 8-byte local access per push
    // and per pop.
    uint2 stack[kTerrainStack];
    stack[0] = make_uint2(0u, __float_as_uint(fmaxf(root.x, 0.0f)));
    uint32_t count = 1u;
    while (count > 0u) {
        count -= 1u;
        const uint2 top = stack[count];
        if (__uint_as_float(top.y) >= limit) continue;
        uint32_t index = top.x;
        for (;;) {
            // The node's size from its heap level; its cell coordinates (the
            // Morton decode of t_node) only where a leaf needs them.
            const uint32_t size = cells >> ((31u - __clz(3u * index + 1u)) / 2u);
            if (size == 2u) {
                const uint3 node = t_node(index, cells);
                // On compact grids a vertex's x and z come from its indices:
                // the leaf's three columns and rows once, not per triangle.
                const bool compact = t_compact(cells);
                float cx[3] = {0.0f, 0.0f, 0.0f}, cz[3] = {0.0f, 0.0f, 0.0f};
                if (compact) {
#pragma unroll
                    for (uint32_t k = 0; k < 3u; ++k) {
                        cx[k] = t_coordinate(node.x + k, cells, scale);
                        cz[k] = t_coordinate(node.y + k, cells, scale);
                    }
                }
#pragma unroll 1
                for (uint32_t z = node.y; z < node.y + 2u; ++z) {
#pragma unroll 1
                    for (uint32_t x = node.x; x < node.x + 2u; ++x) {
                        if constexpr (C) ev->terrain_triangles += 2u;
                        float3 a, b, c, e;
                        if (compact) {
                            const bool x1 = x != node.x, z1 = z != node.y;
                            const float x0c = x1 ? cx[1] : cx[0], x1c = x1 ? cx[2] : cx[1];
                            const float z0c = z1 ? cz[1] : cz[0], z1c = z1 ? cz[2] : cz[1];
                            a = f3(x0c, t_height(T, cells, x, z), z0c);
                            b = f3(x1c, t_height(T, cells, x + 1u, z), z0c);
                            c = f3(x0c, t_height(T, cells, x, z + 1u), z1c);
                            e = f3(x1c, t_height(T, cells, x + 1u, z + 1u), z1c);
                        } else {
                            a = t_vertex(T, cells, scale, x, z);
                            b = t_vertex(T, cells, scale, x + 1u, z);
                            c = t_vertex(T, cells, scale, x, z + 1u);
                            e = t_vertex(T, cells, scale, x + 1u, z + 1u);
                        }
                        const float3 first = t_triangle(o, d, a, c, b);
                        const float3 second = t_triangle(o, d, e, b, c);
                        if (first.z < limit) {
                            if (occlusion) return make_float4(0.0f, 0.0f, 0.0f, first.z);
                            float3 n = normalize(t_normal(T, cells, x, z) * (1.0f - first.x - first.y) +
                                                 t_normal(T, cells, x, z + 1u) * first.x +
                                                 t_normal(T, cells, x + 1u, z) * first.y);
                            if (alpine) n = style::alpine_face_shading(n, a, c, b);
                            result = make_float4(n.x, n.y, n.z, first.z);
                            limit = first.z;
                        }
                        if (second.z < limit) {
                            if (occlusion) return make_float4(0.0f, 0.0f, 0.0f, second.z);
                            float3 n = normalize(t_normal(T, cells, x + 1u, z + 1u) * (1.0f - second.x - second.y) +
                                                 t_normal(T, cells, x + 1u, z) * second.x +
                                                 t_normal(T, cells, x, z + 1u) * second.y);
                            if (alpine) n = style::alpine_face_shading(n, e, b, c);
                            result = make_float4(n.x, n.y, n.z, second.z);
                            limit = second.z;
                        }
                    }
                }
                break;
            }
            if constexpr (C) ev->terrain_nodes += 1u;
            uint32_t children[4];
            float distances[4];
            const float4 *box = reinterpret_cast<const float4 *>(T + t_cache(cells) + (size_t)(index * 4u + 1u) * 6u);
            const float4 q0 = box[0], q1 = box[1], q2 = box[2], q3 = box[3], q4 = box[4], q5 = box[5];
            const float3 lo[4] = {f3(q0.x, q0.y, q0.z), f3(q1.z, q1.w, q2.x), f3(q3.x, q3.y, q3.z), f3(q4.z, q4.w, q5.x)};
            const float3 hi[4] = {f3(q0.w, q1.x, q1.y), f3(q2.y, q2.z, q2.w), f3(q3.w, q4.x, q4.y), f3(q5.y, q5.z, q5.w)};
#pragma unroll
            for (uint32_t child = 0; child < 4u; ++child) {
                children[child] = index * 4u + child + 1u;
                const float2 bounds = t_interval(lo[child], hi[child], o, inv);
                distances[child] =
                    (bounds.x <= bounds.y && bounds.y > 0.001f && bounds.x < limit) ? fmaxf(bounds.x, 0.0f) : 1.0e30f;
            }
            // Far first on the stack; the nearest child is visited next.
            // The reference's insertion sort, as a fixed sequence of
            // compare-exchanges that swap only on a strictly nearer left
            // element: once an element stops, the ones before it are no
            // nearer, so the extra exchanges never fire and the order
            // (ties included) is the insertion sort's.
#pragma unroll
            for (uint32_t i = 1; i < 4u; ++i) {
#pragma unroll
                for (uint32_t j = i; j > 0u; --j) {
                    const bool swap = distances[j - 1u] < distances[j];
                    const float dl = distances[j - 1u], dr = distances[j];
                    const uint32_t cl = children[j - 1u], cr = children[j];
                    distances[j - 1u] = swap ? dr : dl;
                    distances[j] = swap ? dl : dr;
                    children[j - 1u] = swap ? cr : cl;
                    children[j] = swap ? cl : cr;
                }
            }
#pragma unroll
            for (uint32_t i = 0; i < 3u; ++i) {
                if (distances[i] < limit && count < (uint32_t)kTerrainStack) {
                    stack[count] = make_uint2(children[i], __float_as_uint(distances[i]));
                    count += 1u;
                }
            }
            // The nearest child would be pushed last and popped at once
            // with the same limit: descend into it directly.
            if (!(distances[3] < limit && count < (uint32_t)kTerrainStack)) break;
            index = children[3];
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
// A rock (kinds 2, 2.25) or vegetation (3 conifer, 4 grass, 5 trunk;
// forest.wgsl:56-136): one out-of-line call site in the primitive loop.
static __device__ __noinline__ float4 solid_hit(float kind, float3 p, float3 v, float3 e) {
    if (kind > 2.5f) {
        const style::veg_hit g =
            style::vegetation_hit(kind, style::V(p.x, p.y, p.z), style::V(v.x, v.y, v.z), style::V(e.x, e.y, e.z));
        return make_float4(g.n.x.v, g.n.y.v, g.n.z.v, g.t.v);
    }
    return rock_hit(p, v, e);
}

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
        const float4 terrain = terrain_query<C>(S.p->terrain, S.p->terrain_cells, radius,
                                                (S.s->g.ground_counts[2] & 255u) == 3u, o, d, tl, occlusion, K.ev);
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
            K.add(&Events::prop_boxes);
            const float2 bounds = box_interval(sub_rn(o, center), d, e);
            if (bounds.x > bounds.y || bounds.y <= 0.001f || __fdiv_rn(bounds.x, kMetresPerAu) > closest.t)
                i += (uint32_t)(-kind);
            continue;
        }
        K.add(&Events::prop_tests);
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
            // Rocks and vegetation, inside their bounding boxes.
            const float2 bounds = box_interval(p, v, e);
            if (bounds.x > bounds.y || bounds.y <= 0.001f || __fdiv_rn(bounds.x, kMetresPerAu) > closest.t) continue;
            const float4 solid = solid_hit(kind, p, v, e);
            distance = solid.w;
            n = xyz(solid);
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

namespace style {

// Landscape themes 3 (alpine) and 5 (dunes), in the strict arithmetic of
// the surface styles (sg_surface.cuh): their floors hash surface-frame
// coordinates, so each operation rounds exactly as the CPU restatement's.
struct v2 {
    sf x, y;
};
__device__ __forceinline__ v2 V2(sf x, sf y) { return v2{x, y}; }
__device__ __forceinline__ sf v2dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ sf v2len(v2 a) { return sqrtf(a.x * a.x + a.y * a.y); }
__device__ __forceinline__ sv to_ground_s(const Scene &S, sv v) {
    const float3 g = to_ground(S, to_f3(v));
    return V(g.x, g.y, g.z);
}
__device__ __forceinline__ sv from_ground_s(const Scene &S, sv v) {
    const float3 g = from_ground(S, to_f3(v));
    return V(g.x, g.y, g.z);
}
__device__ __forceinline__ sf terrain_scale(const Scene &S) {
    return clampf_(sf(S.s->g.ground_up[3]) / sf(200000.0f), 0.0001f, 1.0f);
}
__device__ __forceinline__ sf footprint_at(const Scene &S, sf distance) {
    return distance * 2.0f * S.s->g.cam_forward[3] / maxf_(S.s->g.viewport[1], 1.0f);
}
// The surface-frame point in terrain units above the curved datum.
__device__ __forceinline__ sv terrain_local(const Scene &S, sv p) {
    const sf c = sf(t_curvature(p.x.v, p.z.v, S.s->g.ground_up[3]));
    return vdivs(V(p.x, p.y - c, p.z), terrain_scale(S));
}

/* ---------------------------------------------------------------- */
/* Landscape themes 3 (alpine) and 5 (dunes): ground.wgsl:320-596,   */
/* terrain.wgsl:142-150. Strict f32 with correctly rounded            */
/* transcendentals, like the surface styles.                          */
/* ---------------------------------------------------------------- */
constexpr float ICE_FLOW = 4.4f;
constexpr float DUNE_WIND = 0.61f;
constexpr float DUNE_PAN_LEVEL = 2.0f;

/* lookout_hill: ground.wgsl:322-325 */
static __device__ __noinline__ sf lookout_hill(sf r) {
    sf u = minf_(v2len(V2(r, 30.0f)) / 700.0f, 1.0f);
    return 180.0f * (1.0f - u) * (1.0f - u);
}

/* dune_cracks: ground.wgsl:490-503 (the gap between the two nearest
 * jittered cells). */
static __device__ __noinline__ sf dune_cracks(v2 p) {
    v2 g = V2(floorf(p.x), floorf(p.y));
    v2 f = V2(p.x - g.x, p.y - g.y);
    sf d1 = 8.0f, d2 = 8.0f;
    for (int j = -1; j <= 1; j++) {
        for (int i = -1; i <= 1; i++) {
            v2 o = V2((float)i, (float)j);
            sv h = hash33(V(g.x + o.x, g.y + o.y, 3.0f));
            sf d = v2len(V2(o.x + 0.15f + 0.7f * h.x - f.x, o.y + 0.15f + 0.7f * h.y - f.y));
            if (d < d1) {
                d2 = d1;
                d1 = d;
            } else if (d < d2) {
                d2 = d;
            }
        }
    }
    return d2 - d1;
}

/* ice_crevasse: ground.wgsl:333-360; (coverage, depth from the lip). */
static __device__ __noinline__ v2 ice_crevasse(v2 q, sf footprint) {
    sf r = v2len(q);
    sf tension = smoothstepf(650.0f, 900.0f, r) * (1.0f - smoothstepf(1800.0f, 2600.0f, r));
    sf strain = maxf_(smoothstepf(0.47f, 0.58f, fbm(V(q.x / 2600.0f + 4.0f, 2.0f, q.y / 2600.0f), 2)), tension) *
                   smoothstepf(600.0f, 750.0f, r);
    if (strain <= 0.0f) return V2(0.0f, 0.0f);
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    sf along = v2dot(q, flow) + 280.0f * (vnoise(V(q.x / 1500.0f, q.y / 1500.0f, 1.0f)) - 0.5f);
    sf across = v2dot(q, V2(flow.y, -flow.x)) + 120.0f * (vnoise(V(q.x / 900.0f, q.y / 900.0f, 5.0f)) - 0.5f);
    sf spacing = 60.0f;
    sf row = floorf(along / spacing);
    uint32_t key = hash_u32(((uint32_t)(int32_t)row.v * 0x8da6b343u) ^ 0xc3e5u);
    sf length_m = 120.0f + 300.0f * (float)(key & 255u) / 255.0f;
    sf s = across / length_m + (float)((key >> 8u) & 255u) / 255.0f;
    sf segment = floorf(s);
    sf lens = pow_d(maxf_(sin_d(PI_F * (s - segment)), 0.0f), 0.7f);
    uint32_t open = hash_u32(key ^ (uint32_t)(int32_t)segment.v);
    if ((open & 255u) < 70u) return V2(0.0f, 0.0f);
    sf centre = 0.5f + 0.3f * ((float)((open >> 8u) & 255u) / 255.0f - 0.5f);
    sf half_width = 0.5f * (2.0f + 14.0f * (float)((open >> 16u) & 255u) / 255.0f) * lens * strain;
    sf d = fabsf(along / spacing - row - centre) * spacing + 0.8f * (vnoise(V(q.x * 0.15f, q.y * 0.15f, 9.0f)) - 0.5f);
    sf aa = maxf_(footprint, 1.0e-3f);
    sf coverage = clampf_((half_width - d) / aa + 0.5f, 0.0f, 1.0f) * minf_(1.0f, 2.0f * half_width / aa);
    return V2(coverage, 1.0f - clampf_(d / maxf_(half_width, 1.0e-3f), 0.0f, 1.0f));
}

/* alpine_floor: ground.wgsl:365-427 */
static __device__ __noinline__ sv alpine_floor(const Scene &S, sv p, sf distance, sv normal) {
    sf scale = terrain_scale(S);
    sv q = terrain_local(S, p);
    sf hill = lookout_hill(v2len(V2(q.x, q.z)));
    q.y = q.y - hill;
    sf footprint = footprint_at(S, distance) / scale;
    sf detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    sf slope = 1.0f - maxf_(normal.y, 0.0f);
    sf broad = vnoise(vadd(vmul(q, 0.004f), V(11.0f, 4.0f, 1.0f)));
    sf middle = vnoise(vmul(q, 0.2f));
    sf grain = vnoise(vmul(q, 4.0f));
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    sf along = v2dot(V2(q.x, q.z), flow);
    sf across = v2dot(V2(q.x, q.z), V2(flow.y, -flow.x));
    sf crust = smoothstepf(0.45f, 0.6f, fbm(V(along * 0.004f, 2.0f, across * 0.012f), 3));
    sv snow = vmix(V(0.86f, 0.88f, 0.91f), V(0.76f, 0.8f, 0.86f), crust);
    snow = vmul(snow, 0.97f + 0.05f * middle);
    sf bare = smoothstepf(0.47f, 0.53f, fbm(vadd(vmul(q, 0.0016f), V(3.0f, 0.0f, 8.0f)), 4) + 0.1f * (broad - 0.5f));
    sv ice = vmix(V(0.36f, 0.55f, 0.7f), V(0.52f, 0.67f, 0.78f), middle);
    sf fracture_width = 0.03f + footprint / 4.0f;
    sf fractures = (1.0f - smoothstepf(0.0f, fracture_width, dune_cracks(V2(q.x / 4.0f + 9.0f, q.z / 4.0f + 9.0f)))) *
                      0.03f / fracture_width;
    ice = vmix(ice, V(0.82f, 0.86f, 0.9f), minf_(fractures, 1.0f) * 0.7f);
    ice = vmul(ice, 1.0f + (grain - 0.5f) * 0.12f * detail);
    sv glacier = vmix(snow, ice, bare);
    sv debris = vmix(V(0.12f, 0.115f, 0.11f), V(0.26f, 0.24f, 0.22f), grain);
    sf dirty = smoothstepf(6.0f, 30.0f, q.y) * (1.0f - smoothstepf(30.0f, 70.0f, q.y));
    glacier = vmix(glacier, vmix(debris, glacier, 0.45f), dirty * smoothstepf(0.4f, 0.7f, broad) * 0.8f);
    sf wall = smoothstepf(0.35f, 0.6f, slope) * (1.0f - smoothstepf(20.0f, 45.0f, q.y));
    sf depth = smoothstepf(4.0f, -4.0f, q.y);
    sv blue = vmix(V(0.32f, 0.55f, 0.72f), V(0.1f, 0.25f, 0.42f), depth);
    glacier = vmix(glacier, vmul(blue, 0.9f + 0.2f * middle), wall);
    v2 crack = ice_crevasse(V2(q.x, q.z), footprint);
    sf fade = 1.0f - smoothstepf(10.0f, 25.0f, q.y);
    crack = V2(crack.x * fade, crack.y * fade);
    sf lip = (1.0f - smoothstepf(0.0f, 0.12f, crack.y)) * crack.x;
    sv inside = vmix(V(0.3f, 0.55f, 0.74f), V(0.02f, 0.06f, 0.12f), smoothstepf(0.1f, 0.8f, crack.y));
    glacier = vmix(glacier, inside, crack.x);
    glacier = vmix(glacier, V(0.9f, 0.92f, 0.95f), lip * 0.5f);
    sf mountain = maxf_(smoothstepf(25.0f, 70.0f, q.y + 30.0f * (broad - 0.5f)), smoothstepf(4.0f, 15.0f, hill));
    sf joints = 1.0f - smoothstepf(0.0f, 0.06f + footprint / 3.0f,
                                      dune_cracks(V2((q.x + q.y * 0.5f) / 3.0f, q.z / 3.0f)));
    sv granite = vmix(V(0.09f, 0.085f, 0.08f), V(0.24f, 0.215f, 0.19f), broad);
    granite = vmul(granite, 0.85f + 0.3f * middle - 0.35f * joints * (1.0f - smoothstepf(0.1f, 1.0f, footprint)));
    sf lichen = smoothstepf(0.68f, 0.78f, vnoise(vmul(q, 0.9f))) * (1.0f - smoothstepf(0.6f, 0.9f, slope));
    granite = vmix(granite, V(0.3f, 0.17f, 0.06f), lichen * 0.5f * detail);
    sf cover = 1.0f - smoothstepf(0.17f, 0.33f, slope + (broad - 0.5f) * 0.18f + (middle - 0.5f) * 0.08f);
    sf scoured = smoothstepf(0.52f, 0.62f, fbm(vadd(vmul(q, 0.012f), V(2.0f, 0.0f, 6.0f)), 4)) *
                    smoothstepf(25.0f, 90.0f, hill) * (1.0f - smoothstepf(150.0f, 172.0f, hill));
    sf cover_hill = cover * (1.0f - scoured);
    sv peak = vmix(granite, snow, cover_hill);
    sv color = vmix(glacier, peak, mountain);
    return vmul(color, 1.0f + (grain - 0.5f) * 0.08f * detail);
}

/* alpine_shading_normal: ground.wgsl:430-459 (telescope-space normal in
 * and out, surface-frame point). */
static __device__ __noinline__ sv alpine_shading_normal(const Scene &S, sv p, sf distance, sv normal) {
    sf footprint = footprint_at(S, distance);
    sv n = to_ground_s(S, normal);
    sf snowy = 1.0f - smoothstepf(0.3f, 0.5f, 1.0f - n.y);
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    v2 side = V2(flow.y, -flow.x);
    v2 gradient = V2(0.0f, 0.0f);
    sf scale = 1.2f, strength = 0.2f;
    for (uint32_t octave = 0; octave < 3u; octave++) {
        sf fade = 1.0f - smoothstepf(0.08f * scale, 0.25f * scale, footprint);
        if (fade > 0.0f) {
            sf a = v2dot(V2(p.x, p.z), flow) / (6.0f * scale);
            sf c = v2dot(V2(p.x, p.z), side) / scale;
            sf e = 0.08f;
            sf o = (float)octave * 13.0f;
            sf da = vnoise(V(a + e, o, c)) - vnoise(V(a - e, o, c));
            sf dc = vnoise(V(a, o, c + e)) - vnoise(V(a, o, c - e));
            sf ridge_ = 1.0f + 1.5f * (1.0f - fabsf(vnoise(V(a, o, c)) * 2.0f - 1.0f));
            sf k = strength * fade * ridge_ * scale;
            sf gx = (flow.x * da / (6.0f * scale) + side.x * dc / scale) / (2.0f * e) * k;
            sf gz = (flow.y * da / (6.0f * scale) + side.y * dc / scale) / (2.0f * e) * k;
            gradient = V2(gradient.x + gx, gradient.y + gz);
        }
        scale *= 6.0f;
        strength *= 0.6f;
    }
    gradient = V2(gradient.x * snowy, gradient.y * snowy);
    return vnormalize(vadd(normal, from_ground_s(S, V(-gradient.x, 0.0f, -gradient.y))));
}

/* dune_pan: ground.wgsl:483-486 */
static __device__ __noinline__ sv dune_pan(uint32_t i) {
    return i == 0u ? V(842.6f, 707.1f, 560.0f) : V(4346.7f, 1164.7f, 900.0f);
}

/* dune_floor: ground.wgsl:509-568 */
static __device__ __noinline__ sv dune_floor(const Scene &S, sv p, sf distance, sv normal) {
    sf scale = terrain_scale(S);
    sv q = terrain_local(S, p);
    sf footprint = footprint_at(S, distance) / scale;
    sf detail = 1.0f - smoothstepf(0.02f, 0.15f, footprint);
    sf slope = 1.0f - maxf_(normal.y, 0.0f);
    sf broad = vnoise(vadd(vmul(q, 0.0015f), V(1.0f, 7.0f, 3.0f)));
    sf middle = vnoise(vmul(q, 0.05f));
    sf rise = smoothstepf(6.0f, 160.0f, q.y + 40.0f * (broad - 0.5f));
    sv plinth = vmix(V(0.3f, 0.095f, 0.038f), V(0.36f, 0.12f, 0.045f), broad);
    sv upper = vmix(V(0.42f, 0.155f, 0.06f), V(0.47f, 0.19f, 0.072f), broad);
    sv sand = vmul(vmix(plinth, upper, rise), 0.94f + 0.08f * middle);
    sf flat = v2len(V2(normal.x, normal.z));
    if (flat > 1.0e-3f) {
        v2 down = V2(-normal.x / flat, -normal.z / flat);
        sf across = v2dot(V2(q.x, q.z), V2(-down.y, down.x));
        sf along = v2dot(V2(q.x, q.z), down);
        sf tongues = fbm(V(across * 0.18f, along * 0.012f, 5.0f), 3);
        sf slip = smoothstepf(0.32f, 0.45f, slope);
        sand = vmix(sand, vmul(vmulv(sand, V(1.06f, 1.12f, 1.16f)), 0.86f + 0.28f * tongues), slip);
    }
    sf lag = smoothstepf(0.6f, 0.76f, fbm(vadd(vmulv(q, V(0.013f, 0.0f, 0.004f)), V(9.0f, 0.0f, 2.0f)), 4)) *
                (1.0f - smoothstepf(0.04f, 0.16f, slope)) * (1.0f - smoothstepf(10.0f, 45.0f, q.y));
    sand = vmix(sand, V(0.13f, 0.065f, 0.05f), lag * 0.55f);
    sf corridor = (1.0f - smoothstepf(5.0f, 16.0f, q.y + 6.0f * (broad - 0.5f))) *
                     (1.0f - smoothstepf(0.03f, 0.1f, slope));
    sv gravel = vmix(V(0.39f, 0.21f, 0.115f), V(0.45f, 0.28f, 0.16f), vnoise(vmul(q, 0.3f)));
    sf pebbles = smoothstepf(0.72f, 0.8f, vnoise(vmul(q, 7.0f))) * detail;
    sand = vmix(sand, vmul(gravel, 1.0f - 0.45f * pebbles), corridor * 0.6f);
    sf pan = 0.0f;
    for (uint32_t i = 0; i < 2u; i++) {
        sv c = dune_pan(i);
        pan = maxf_(pan, 1.0f - smoothstepf(c.z * 1.2f, c.z * 1.35f + 140.0f, v2len(V2(q.x - c.x, q.z - c.y))));
    }
    pan *= 1.0f - smoothstepf(DUNE_PAN_LEVEL + 0.25f, DUNE_PAN_LEVEL + 1.5f, q.y);
    if (pan > 0.0f) {
        sf tone = fbm(vadd(vmul(q, 0.012f), V(4.0f, 0.0f, 1.0f)), 4);
        sv clay = vmix(V(0.4f, 0.35f, 0.29f), V(0.6f, 0.56f, 0.49f), smoothstepf(0.3f, 0.7f, tone));
        clay = vmul(clay, 0.82f + 0.18f * smoothstepf(0.35f, 1.0f, pan));
        sf fine_width = 0.04f + footprint / 0.9f;
        sf cracks = (1.0f - smoothstepf(0.0f, fine_width, dune_cracks(V2(q.x / 0.9f, q.z / 0.9f)))) * 0.04f / fine_width;
        sf wide_width = 0.03f + footprint / 6.0f;
        sf large = (1.0f - smoothstepf(0.0f, wide_width, dune_cracks(V2(q.x / 6.0f + 17.0f, q.z / 6.0f + 17.0f)))) *
                      0.03f / wide_width;
        clay = vmul(clay, 1.0f - 0.6f * minf_(cracks, 1.0f) - 0.45f * minf_(large, 1.0f));
        clay = vmul(clay, 0.92f + 0.16f * vnoise(vmul(q, 2.3f)) * (1.0f - smoothstepf(0.04f, 0.25f, footprint)));
        sand = vmix(sand, clay, pan);
    }
    return vmul(sand, 1.0f + (vnoise(vmul(q, 9.0f)) - 0.5f) * 0.12f * detail);
}

/* dune_ripples: ground.wgsl:571-582; the surface-frame (x, z) gradient. */
static __device__ __noinline__ v2 dune_ripples(sv p, sf wavelength, sf warp, sf amplitude) {
    v2 wind = V2(sin_d(DUNE_WIND), cos_d(DUNE_WIND));
    v2 side = V2(wind.y, -wind.x);
    sf bend = warp * (vnoise(V(p.x / (9.0f * wavelength), p.z / (9.0f * wavelength), 1.0f)) +
                         0.35f * vnoise(V(p.x / (2.5f * wavelength), p.z / (2.5f * wavelength), 7.0f)));
    sf phase = v2dot(V2(p.x, p.z), wind) / wavelength + bend +
                  0.4f * sin_d(v2dot(V2(p.x, p.z), side) / (3.0f * wavelength));
    sf theta = TAU_F * phase;
    sf slope = cos_d(theta + 0.65f * sin_d(theta)) * (1.0f + 0.65f * cos_d(theta));
    sf patches = smoothstepf(0.25f, 0.6f, vnoise(V(p.x / (14.0f * wavelength), p.z / (14.0f * wavelength), 3.0f)));
    sf k = slope * amplitude * TAU_F / wavelength * patches;
    return V2(wind.x * k, wind.y * k);
}

/* dune_shading_normal: ground.wgsl:583-595 */
static __device__ __noinline__ sv dune_shading_normal(const Scene &S, sv p, sf distance, sv normal) {
    sf footprint = footprint_at(S, distance);
    sv n = to_ground_s(S, normal);
    sf gentle = 1.0f - smoothstepf(0.22f, 0.38f, 1.0f - n.y);
    sv q = terrain_local(S, p);
    sf dry = smoothstepf(DUNE_PAN_LEVEL + 0.4f, DUNE_PAN_LEVEL + 1.5f, q.y);
    v2 gradient = V2(0.0f, 0.0f);
    sf fine = 1.0f - smoothstepf(0.03f, 0.07f, footprint);
    if (fine > 0.0f) {
        v2 r = dune_ripples(p, 0.12f, 2.5f, 0.006f);
        gradient = V2(gradient.x + r.x * fine, gradient.y + r.y * fine);
    }
    sf coarse = (1.0f - smoothstepf(0.15f, 0.4f, footprint)) * (1.0f - smoothstepf(9.0f, 16.0f, q.y));
    if (coarse > 0.0f) {
        v2 r = dune_ripples(vadds(p, 31.0f), 0.8f, 2.0f, 0.03f);
        gradient = V2(gradient.x + r.x * coarse, gradient.y + r.y * coarse);
    }
    sf k = gentle * dry;
    gradient = V2(gradient.x * k, gradient.y * k);
    return vnormalize(vadd(normal, from_ground_s(S, V(-gradient.x, 0.0f, -gradient.y))));
}

// Theme 4 (basalt): the measured elevation atlas follows the terrain's
// vertex cache; reads past the uploaded atlas return 0.
__device__ __forceinline__ uint32_t u32_sat(float x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967040.0f) return 0xffffffffu;
    return (uint32_t)x;
}
__device__ __forceinline__ int32_t i32_sat(float x) {
    if (!(x > -2147483520.0f)) return x != x ? 0 : (int32_t)0x80000000u;
    if (x >= 2147483520.0f) return 0x7fffffff;
    return (int32_t)x;
}
__device__ __forceinline__ sf fract_(sf x) { return x - floorf(x); }
__device__ __forceinline__ sf log2_d(sf x) { return sf((float)::log2((double)x.v)); }
__device__ __forceinline__ sf volcano_data(const Scene &S, uint32_t i) {
    if (!S.p->terrain || i >= S.p->terrain_detail_floats) return sf(0.0f);
    const uint32_t cells = S.p->terrain_cells;
    return sf(S.p->terrain[(size_t)t_vertex_cache(cells) + (size_t)t_vertices(cells) * t_vertex_stride(cells) + i]);
}
struct v4 {
    sf x, y, z, w;
};
__device__ __forceinline__ v4 volcano_record(const Scene &S, uint32_t i) {
    return v4{volcano_data(S, i), volcano_data(S, i + 1u), volcano_data(S, i + 2u), volcano_data(S, i + 3u)};
}
/* ---------------------------------------------------------------- */
/* Theme 4 (basalt): basalt_floor (ground.wgsl:463-477) and the      */
/* shading normals from the measured elevation atlas that follows the */
/* terrain's vertex cache (volcano.wgsl). Reads past the uploaded     */
/* atlas return 0 (the reference's buffer always holds one).          */
/* ---------------------------------------------------------------- */
__device__ __forceinline__ uint32_t clamp_index(int32_t v, uint32_t width) {
    int32_t hi = (int32_t)width - 1;
    return (uint32_t)(v < 0 ? 0 : (v > hi ? hi : v));
}
static __device__ __noinline__ sf volcano_bilinear(const Scene &S, uint32_t offset, uint32_t width, v2 uv) {
    v2 pixel = V2(uv.x * (float)width - 0.5f, uv.y * (float)width - 0.5f);
    int32_t lx = i32_sat(floorf(pixel.x).v), ly = i32_sat(floorf(pixel.y).v);
    uint32_t ax = clamp_index(lx, width), ay = clamp_index(ly, width);
    uint32_t bx = clamp_index(lx == 0x7fffffff ? lx : lx + 1, width), by = clamp_index(ly == 0x7fffffff ? ly : ly + 1, width);
    v2 f = V2(fract_(pixel.x), fract_(pixel.y));
    return mixf(mixf(volcano_data(S, offset + ay * width + ax), volcano_data(S, offset + ay * width + bx), f.x),
                mixf(volcano_data(S, offset + by * width + ax), volcano_data(S, offset + by * width + bx), f.x), f.y);
}
static __device__ __noinline__ sf volcano_map(const Scene &S, uint32_t map, v2 p, sf footprint) {
    v4 desc = volcano_record(S, map * 4u);
    v2 local = V2(p.x, p.y - desc.w);
    sf reach = 0.5f * (desc.y - 1.0f) * desc.z;
    if (fabsf(local.x) > reach || fabsf(local.y) > reach) return 0.0f;
    v2 uv = V2((local.x / desc.z + 0.5f * desc.y) / desc.y, (local.y / desc.z + 0.5f * desc.y) / desc.y);
    sf lod = maxf_(log2_d(maxf_(footprint / desc.z, 1.0f)), 0.0f);
    uint32_t offset = u32_sat(desc.x.v), width = u32_sat(desc.y.v);
    uint32_t levels = u32_sat(lod.v);
    for (uint32_t level = 0; level < levels && width > 1u; level++) {
        offset += width * width;
        width = (width + 1u) / 2u;
    }
    sf a = volcano_bilinear(S, offset, width, uv);
    if (width == 1u) return a;
    sf b = volcano_bilinear(S, offset + width * width, (width + 1u) / 2u, uv);
    return mixf(a, b, fract_(lod));
}
static __device__ __noinline__ sf volcano_fine_weight(const Scene &S, v2 p) {
    v4 desc = volcano_record(S, 4u);
    v2 local = V2(p.x, p.y - desc.w);
    sf reach = 0.5f * (desc.y - 1.0f) * desc.z;
    return 1.0f - smoothstepf(reach - 72.0f, reach, maxf_(fabsf(local.x), fabsf(local.y)));
}
static __device__ __noinline__ sf volcano_height(const Scene &S, uint32_t map, v2 p, sf footprint) {
    sf coarse = volcano_map(S, map, p, footprint);
    if (map != 0u) return coarse;
    sf weight = volcano_fine_weight(S, p);
    if (weight <= 0.0f) return coarse;
    return mixf(coarse, volcano_map(S, 1u, p, footprint), weight);
}
/* volcano_normal: volcano.wgsl:49-88 (surface-frame normals). */
static __device__ __noinline__ sv volcano_normal(const Scene &S, sv p, sf distance, sv fallback) {
    sf scale = terrain_scale(S);
    v2 point = V2(p.x / scale, p.z / scale);
    sf footprint = footprint_at(S, distance) / scale;
    sf best = 1.0f;
    uint32_t chosen = 0u;
    v2 local = V2(0.0f, 0.0f);
    v4 transform = {0.0f, 0.0f, 1.0f, 0.0f};
    sf site_scale = 1.0f;
    for (uint32_t site = 0; site < 9u; site++) {
        v4 frame = volcano_record(S, 16u + site * 8u);
        v4 info = volcano_record(S, 20u + site * 8u);
        v2 relative = V2((point.x - frame.x) / info.x, (point.y - frame.y) / info.x);
        v2 q = V2(frame.z * relative.x - frame.w * relative.y, frame.w * relative.x + frame.z * relative.y);
        sf height = volcano_height(S, u32_sat(info.y.v), q, footprint / info.x) * info.x;
        if (height > best) {
            best = height;
            chosen = u32_sat(info.y.v);
            local = q;
            transform = frame;
            site_scale = info.x;
        }
    }
    if (best <= 1.0f) return fallback;
    sf spacing = volcano_record(S, chosen * 4u).z;
    if (chosen == 0u) spacing = mixf(spacing, 1.0f, volcano_fine_weight(S, local));
    sf delta = maxf_(spacing, footprint / site_scale * 0.5f);
    sf fp = footprint / site_scale;
    sf dx = (volcano_height(S, chosen, V2(local.x + delta, local.y), fp) -
                volcano_height(S, chosen, V2(local.x - delta, local.y), fp)) / (2.0f * delta);
    sf dz = (volcano_height(S, chosen, V2(local.x, local.y + delta), fp) -
                volcano_height(S, chosen, V2(local.x, local.y - delta), fp)) / (2.0f * delta);
    v2 gradient = V2(transform.z * dx + transform.w * dz, -transform.w * dx + transform.z * dz);
    sf radius = S.s->g.ground_up[3];
    sf k = sqrtf(maxf_(radius * radius - (p.x * p.x + p.z * p.z), 1.0f));
    v2 curvature = V2(p.x / k, p.z / k);
    sv n = vnormalize(V(-gradient.x + curvature.x, 1.0f, -gradient.y + curvature.y));
    if (vdot(n, fallback) < 0.2f) return vnormalize(vmix(fallback, n, 0.7f));
    return n;
}

/* basalt_floor: ground.wgsl:463-477 */
static __device__ __noinline__ sv basalt_floor(const Scene &S, sv p, sf distance, sv normal) {
    sf footprint = footprint_at(S, distance);
    sf broad = fbm(vadd(vmul(p, 0.006f), V(5.0f, 9.0f, 2.0f)), 4);
    sf weather = fbm(vadd(vmul(p, 0.017f), V(23.0f, 7.0f, 11.0f)), 3);
    sf middle = mixf(fbm(vmul(p, 0.08f), 3), 0.5f, smoothstepf(1.0f, 12.0f, footprint));
    sv ash = vmix(V(0.065f, 0.060f, 0.052f), V(0.14f, 0.12f, 0.095f), broad);
    sv rock = vmix(V(0.028f, 0.030f, 0.031f), V(0.07f, 0.064f, 0.054f), middle);
    rock = vmix(rock, V(0.16f, 0.073f, 0.037f), smoothstepf(0.48f, 0.68f, weather) * 0.45f);
    sf slope = 1.0f - maxf_(normal.y, 0.0f);
    sf loose = 1.0f - smoothstepf(0.14f, 0.43f, slope + 0.12f * (weather - 0.5f));
    sv color = vmix(rock, ash, loose);
    color = vmul(color, 0.86f + 0.28f * middle);
    sf grain = vnoise(vmul(p, 5.0f));
    return vmul(color, 1.0f + (grain - 0.5f) * 0.28f * (1.0f - smoothstepf(0.025f, 0.2f, footprint)));
}

}  // namespace style

// Albedo-map extension: index of the nearest texel at surface-frame (x, z).
__device__ __forceinline__ uint32_t map_texel(const TraceParams *P, float3 p) {
    const float u = (p.x / P->map_extent + 1.0f) * 0.5f * (float)P->map_width;
    const float w = (p.z / P->map_extent + 1.0f) * 0.5f * (float)P->map_height;
    int i = (int)floorf(u), j = (int)floorf(w);
    i = max(0, min(i, (int)P->map_width - 1));
    j = max(0, min(j, (int)P->map_height - 1));
    return (uint32_t)j * P->map_width + (uint32_t)i;
}

// landscape_albedo (ground.wgsl:597-632), themes 0-5, plus the map.
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
        if (theme >= 3u && theme <= 5u) {
            const style::sv sp = style::V(p.x, p.y, p.z), sn = style::V(n.x, n.y, n.z);
            if (theme == 3u) return style::to_f3(style::alpine_floor(S, sp, distance, sn));
            if (theme == 4u) return style::to_f3(style::basalt_floor(S, sp, distance, sn));
            return style::to_f3(style::dune_floor(S, sp, distance, sn));
        }
        return forest_floor(p, footprint, n);
    }
    const float4 albedo = S.p->props[3u * (index - kLocalBase - 1u) + 2u];
    const float3 tint = xyz(albedo);
    const float kind = albedo.w;
    if (kind == 0.0f) return tint;
    const float middle = vnoise(p * 1.7f);
    const float fine = mixf(vnoise(p * 12.0f), 0.5f, smoothstepf(18.0f, 110.0f, distance));
    if (kind > 4.5f) return tint * (0.65f + 0.6f * middle);
    if (kind > 2.5f) {
        // Conifers: bark on the lower trunk (ground.wgsl:618-625).
        const uint32_t k = index - kLocalBase - 1u;
        const float4 oc = S.p->props[3u * k], oe = S.p->props[3u * k + 1u];
        const float4 t1 = S.p->prop_trig[2u * k + 1u];
        const float3 q = div3_rn(rotate_north(sub_rn(p, xyz(oc)), -t1.x, t1.y), xyz(oe));
        if (kind > 3.5f || (q.y < -0.35f && __fsqrt_rn(__fadd_rn(__fmul_rn(q.x, q.x), __fmul_rn(q.z, q.z))) < 0.09f)) {
            const float bark = vnoise(f3(__fmul_rn(p.x, 25.0f), __fmul_rn(p.y, 1.5f), __fmul_rn(p.z, 25.0f)));
            return f3(0.13f, 0.073f, 0.032f) * (0.5f + 0.85f * bark);
        }
        return tint * (0.7f + 0.55f * middle + 0.2f * fine);
    }
    const float strata = sinf(p.y * 8.0f + 2.5f * middle);
    const float lichen = smoothstepf(0.52f, 0.76f, middle) * fmaxf(n.y, 0.0f);
    const float3 stone = tint * (0.7f + 0.45f * fine + 0.07f * strata);
    if ((S.s->g.ground_counts[2] & 255u) != 0u) return stone;
    return mix3(stone, f3(0.11f, 0.145f, 0.037f), lichen * 0.65f);
}

// landscape_shading_normal (ground.wgsl:633-648), themes 0-5.
static __device__ __noinline__ float3 landscape_shading_normal(Scene S, Ray ray, float t, uint32_t index, float3 normal) {
    if (index != kLocalBase && index != kTerrainId) return normal;
    const float3 p = landscape_point(S, ray, t);
    const float distance = t * kMetresPerAu;
    const uint32_t theme = S.s->g.ground_counts[2] & 255u;
    if (theme == 4u && index == kTerrainId) {
        // The survey's elevations supply the detail (volcano.wgsl).
        const float3 g = to_ground(S, normal);
        const style::sv n = style::volcano_normal(S, style::V(p.x, p.y, p.z), distance, style::V(g.x, g.y, g.z));
        return from_ground(S, style::to_f3(n));
    }
    if (theme == 3u || theme == 5u) {
        const style::sv sp = style::V(p.x, p.y, p.z), sn = style::V(normal.x, normal.y, normal.z);
        return style::to_f3(theme == 5u ? style::dune_shading_normal(S, sp, distance, sn)
                                        : style::alpine_shading_normal(S, sp, distance, sn));
    }
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
