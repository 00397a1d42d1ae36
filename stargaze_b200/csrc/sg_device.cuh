// sg_device.cuh — device-side integrator for the B200 (sm_100a).
//
// Behaviour follows stargaze's progressive integrator:
//   src/shaders/pathtrace.wgsl  (sample loop, spheres, stellar NEE + MIS,
//                                ringshine, point discs, Russian roulette)
//   src/shaders/rings.wgsl      (zero-thickness Beer-Lambert ring slabs)
//
// Design for the B200:
//   * Settings travel as a __grid_constant__ kernel parameter (constant
//     bank, uniform broadcast); the body table (160 B per body) and the ring
//     optical-depth tables are staged once per CTA in shared memory.
//   * The geometric core (sphere and ring intersection distances, the
//     discriminant and the annulus test) is evaluated with explicit
//     round-to-nearest intrinsics, never contracted into FMAs, so hit ids and
//     distances are bit-identical to an IEEE f32 evaluation of the WGSL
//     expressions. Shading arithmetic is free to use FMA.
//   * Closest-hit loops track only (distance, index, root offset); the
//     surface normal is formed once for the winning body.
//   * Instruction footprint: the light-sampling, shadow-ray, slab-BSDF,
//     ringshine and point-disc helpers are out of line so their several call
//     sites share one copy (divergent warps otherwise stall on instruction
//     fetch). They take and return values only — nothing whose address
//     escapes — so calls cost no local memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/stargaze_b200.h"
#include "sg_internal.h"

// Call attribute of the multi-site helpers (sample_light, light_visibility,
// ring_bsdf, ringshine, point_disc_hit): out of line by default.
#ifndef SG_HELPER
#define SG_HELPER __noinline__
#endif

namespace sg {

constexpr float kPi = 3.141592653589793f;
constexpr float kTau = 6.283185307179586f;
constexpr uint32_t kMiss = SG_MISS;
constexpr float kStarDotPixels = 3.0f;
constexpr float kPointDiscRadius = 0.00136f;
constexpr float kRingIndirectCap = 0.003f;
constexpr int kBodyVec4 = 10;  // float4 words per sg_sphere

// Field order inside one staged body (pathtrace.wgsl:26-37).
enum BodyField : int {
    kCenter = 0,      // xyz high part, w radius
    kMaterial = 1,    // rgb, w emissive
    kLow = 2,         // xyz low part, w mottle strength
    kRingPlane = 3,   // pole, inner
    kRingParams = 4,  // outer, tau, banded, table slot + 1
    kRingColor = 5,
    kAxisX = 6,          // xyz body X axis, w surface style
    kAxisY = 7,          // xyz body Y axis, w pattern seed
    kSurfaceColor = 8,   // secondary colour, w turbulence or crater density
    kSurfaceParams = 9,  // bands, storms or ice caps, ocean, clouds
};

// ---------------------------------------------------------------------------
// float3 algebra
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float3 normalize(float3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
__device__ __forceinline__ float length(float3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ float luminance(float3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
__device__ __forceinline__ float max3(float3 v) { return fmaxf(v.x, fmaxf(v.y, v.z)); }
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
    float t = clampf((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}

// Strict (never contracted) forms for the geometric core.
__device__ __forceinline__ float3 add_rn(float3 a, float3 b) {
    return f3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
}
__device__ __forceinline__ float3 sub_rn(float3 a, float3 b) {
    return f3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
}
__device__ __forceinline__ float3 mul_rn(float3 a, float s) {
    return f3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s));
}
__device__ __forceinline__ float dot_rn(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 cross_rn(float3 a, float3 b) {
    return f3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
              __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
              __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float3 div_rn(float3 a, float s) {
    return f3(__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s));
}
__device__ __forceinline__ float length_rn(float3 a) { return __fsqrt_rn(dot_rn(a, a)); }

// sin and cos of 2*pi*u for u in [0, 1): sincospif needs no Payne-Hanek
// range reduction, so the code stays small and branch-free.
__device__ __forceinline__ void sincos_turn(float u, float *s, float *c) { sincospif(2.0f * u, s, c); }

// ---------------------------------------------------------------------------
// RNG (pathtrace.wgsl:87-98): PCG-style LCG step with a 24-bit output.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
    x = (x ^ (x >> 16)) * 0x7feb352du;
    x = (x ^ (x >> 15)) * 0x846ca68bu;
    return x ^ (x >> 16);
}

// Event counters for the algorithmic-work model.
struct Events {
    uint32_t vertices, sphere_tests, sphere_hits, ring_tests, light_samples, shadow_rays,
        ring_events, surface_events, rng_draws, terrain_nodes, terrain_triangles, prop_boxes, prop_tests;
};

// Counting is compiled out of the production variant (C == false); L turns
// the local landscape on, F the FP64 sites (sg_set_fp64_sites).
template <bool C, bool L, bool F>
struct Counter {
    Events *ev;
    __device__ __forceinline__ void add(uint32_t Events::*f) const {
        if constexpr (C) ev->*f += 1u;
    }
};

template <bool C, bool L, bool F>
__device__ __forceinline__ float rnd(Counter<C, L, F> K, uint32_t &state) {
    K.add(&Events::rng_draws);
    state = state * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28) + 4u)) ^ state) * 277803737u;
    return (float)(((word >> 22) ^ word) >> 8) * (1.0f / 16777216.0f);
}

// ---------------------------------------------------------------------------
// Scene view inside a CTA
// ---------------------------------------------------------------------------
struct Scene {
    const TraceParams *p;   // the launch's parameters (kernel parameter space)
    const sg_settings *s;   // &p->s
    const float4 *B;        // staged bodies, kBodyVec4 float4 each
    const float *tables;    // ring optical-depth tables (slot-major)
};

struct Ray {
    float3 o;  // offset from bodies[anchor] centre, or camera origin for kMiss
    float3 d;
    uint32_t anchor;
};

__device__ __forceinline__ float4 bf(const Scene &S, uint32_t i, int f) { return S.B[i * kBodyVec4 + f]; }
__device__ __forceinline__ float b_radius(const Scene &S, uint32_t i) { return S.B[i * kBodyVec4 + kCenter].w; }

// relative_center (pathtrace.wgsl:100-113), strict.
__device__ __forceinline__ float3 relative_center(const Scene &S, const Ray &r, uint32_t i) {
    if (r.anchor == i) return -r.o;
    const float3 ci = xyz(bf(S, i, kCenter));
    const float3 li = xyz(bf(S, i, kLow));
    if (r.anchor == kMiss) return add_rn(ci, sub_rn(li, r.o));
    const float3 ca = xyz(bf(S, r.anchor, kCenter));
    const float3 la = xyz(bf(S, r.anchor, kLow));
    return add_rn(sub_rn(ci, ca), sub_rn(sub_rn(li, la), r.o));
}

// Distance part of sphere_hit_radius (pathtrace.wgsl:134-166). Returns the
// hit distance (1e30 on a miss) and the signed root offset `delta` that the
// normal needs.
template <bool C, bool L, bool F>
__device__ __forceinline__ float sphere_distance(const Scene &S, Counter<C, L, F> K, const Ray &r, uint32_t i,
                                                 float radius, float &delta) {
    K.add(&Events::sphere_tests);
    const float3 oc = relative_center(S, r, i);
    const float b = dot_rn(oc, r.d);
    const float c = __fsub_rn(dot_rn(oc, oc), __fmul_rn(radius, radius));
    // An origin outside the sphere with the centre behind it: both roots
    // are negative whatever h is (q = b - root < 0, so q / a < 0 and
    // c / q < 0), so the exact test below would miss. Signs are exact.
    if (b < 0.0f && c > 0.0f) return 1.0e30f;
    const float a = dot_rn(r.d, r.d);
    const float3 pc = cross_rn(oc, r.d);
    const float h = __fsub_rn(__fmul_rn(__fmul_rn(a, radius), radius), dot_rn(pc, pc));
    if (h < 0.0f) return 1.0e30f;
    const float root = __fsqrt_rn(h);
    const float q = __fadd_rn(b, b >= 0.0f ? root : -root);
    if (q == 0.0f) return 1.0e30f;
    // The far root is divided out only when the near one is behind the
    // origin; the values are those of the WGSL's c/q and q/a.
    float distance = b < 0.0f ? __fdiv_rn(q, a) : __fdiv_rn(c, q);
    float signed_root = -root;
    if (distance <= 0.0f) {
        distance = b < 0.0f ? __fdiv_rn(c, q) : __fdiv_rn(q, a);
        signed_root = root;
    }
    if (distance <= 0.0f) return 1.0e30f;
    delta = __fdiv_rn(signed_root, a);
    K.add(&Events::sphere_hits);
    return distance;
}

// Body-local normal of sphere_hit_radius (pathtrace.wgsl:167-170).
__device__ __forceinline__ float3 sphere_normal(const Scene &S, const Ray &r, uint32_t i, float delta) {
    const float3 oc = relative_center(S, r, i);
    const float a = dot_rn(r.d, r.d);
    const float3 pc = cross_rn(oc, r.d);
    const float3 perpendicular = div_rn(cross_rn(r.d, pc), a);
    return normalize(-perpendicular + r.d * delta);
}

struct Hit {
    float t;
    uint32_t index;
    float delta;  // sphere root offset (body hits)
    float3 n;     // telescope-space normal (local landscape hits)
};

// Result of landscape_query (ground.wgsl:123-242; sg_landscape.cuh).
struct LandHit {
    float t;
    uint32_t index;
    float delta;  // root offset when the distant path returns the host sphere
    float3 n;
};
template <bool C, bool L, bool F>
static __device__ SG_HELPER LandHit landscape_query(Scene S, Counter<C, L, F> K, Ray ray, float limit, bool occlusion);

// Bodies and rings a ray is tested against: a camera ray takes its tile's
// cull masks (TraceParams::camera_cull), every other ray all of them. A
// cleared bit is a test that would miss, so skipping it changes nothing.
struct Cull {
    uint32_t bodies, rings;
    __device__ __forceinline__ bool body(uint32_t i) const { return i >= 32u || ((bodies >> i) & 1u); }
    __device__ __forceinline__ bool ring(uint32_t i) const { return i >= 32u || ((rings >> i) & 1u); }
};
constexpr Cull kTestAll{0xffffffffu, 0xffffffffu};

// closest_hit (pathtrace.wgsl:173-185): every body except the landscape
// host, then the landscape.
template <bool C, bool L, bool F>
__device__ __forceinline__ Hit closest_hit(const Scene &S, Counter<C, L, F> K, const Ray &r, Cull cull = kTestAll) {
    Hit best{1.0e30f, kMiss, 0.0f, f3(0.0f, 0.0f, 0.0f)};
    const uint32_t n = S.s->counts[0];
    const float host = S.s->g.ground_north[3];
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (host == (float)(i + 1u) || !cull.body(i)) continue;
        float delta;
        const float t = sphere_distance(S, K, r, i, b_radius(S, i), delta);
        if (t < best.t) best = Hit{t, i, delta, f3(0.0f, 0.0f, 0.0f)};
    }
    if constexpr (L) {
        if (host != 0.0f) {
            const LandHit local = landscape_query(S, K, r, 1.0e30f, false);
            if (local.t < best.t) best = Hit{local.t, local.index, local.delta, local.n};
        }
    }
    return best;
}

// basis_direction (pathtrace.wgsl:187-194).
__device__ __forceinline__ float3 basis_direction(float3 axis, float x, float y, float z) {
    const float3 helper = fabsf(axis.z) > 0.9f ? f3(0.0f, 1.0f, 0.0f) : f3(0.0f, 0.0f, 1.0f);
    const float3 tangent = normalize(cross(helper, axis));
    return normalize(tangent * x + cross(axis, tangent) * y + axis * z);
}

// cone_width (pathtrace.wgsl:197-202): 1 - cos(theta_max) without cancellation.
__device__ __forceinline__ float cone_width_oc(float3 oc, float r) {
    const float sin2 = clampf(r * r / dot(oc, oc), 1.0e-20f, 1.0f);
    return sin2 / (1.0f + sqrtf(1.0f - sin2));
}

__device__ __forceinline__ uint32_t light_count(const sg_settings *s) {
    return s->lights[3] <= 3u ? s->lights[3] : s->counts[0];
}
__device__ __forceinline__ uint32_t light_index(const sg_settings *s, uint32_t slot) {
    return s->lights[3] <= 3u ? s->lights[slot] : slot;
}

struct LightSample {
    float3 d;
    float pdf;
    uint32_t rng;  // the state after the two draws
};

// sample_light (pathtrace.wgsl:214-234), one stratum: uniform cone sampling.
template <bool C, bool L, bool F>
static __device__ SG_HELPER LightSample sample_light(Scene S, Counter<C, L, F> K, Ray r, uint32_t i, uint32_t rng) {
    K.add(&Events::light_samples);
    const float3 oc = relative_center(S, r, i);
    const float3 axis = normalize(oc);
    const float width = cone_width_oc(oc, b_radius(S, i));
    const float radial = rnd(K, rng);
    const float azimuth = rnd(K, rng);
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

// power_weight (pathtrace.wgsl:264-267): power heuristic, beta = 2.
__device__ __forceinline__ float power_weight(float a, float b) {
    const float ratio = b / fmaxf(a, 1.0e-30f);
    return 1.0f / (1.0f + ratio * ratio);
}

// ---------------------------------------------------------------------------
// Rings (rings.wgsl)
// ---------------------------------------------------------------------------
struct RingHit {
    float t;
    uint32_t index;
    float3 p;  // planet-local point
};

__device__ __forceinline__ bool has_ring(const Scene &S, uint32_t i) {
    const float4 rp = bf(S, i, kRingParams);
    return !(rp.x <= bf(S, i, kRingPlane).w || rp.y <= 0.0f);
}

// ---------------------------------------------------------------------------
// FP64 sites (extension, sg_set_fp64_sites): the ring-plane intersection, the
// host-sphere intersection of the landscape and the 5 mm bounce offset
// evaluated in double from the same f32 inputs. Off by default: the f32
// forms are the reference's arithmetic.
// ---------------------------------------------------------------------------
struct d3 {
    double x, y, z;
};
__device__ __forceinline__ d3 D(float3 v) { return d3{(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ d3 operator+(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 operator-(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 operator*(d3 a, double s) { return d3{a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float3 F(d3 v) { return f3((float)v.x, (float)v.y, (float)v.z); }

// ring_hit in double: the centre difference from the hi/lo parts, the
// perpendicular, the plane distance and the annulus test.
static __device__ __noinline__ RingHit ring_hit_fp64(Scene S, Ray r, uint32_t i) {
    const RingHit miss{1.0e30f, kMiss, f3(0.0f, 0.0f, 0.0f)};
    const float4 plane = bf(S, i, kRingPlane);
    const float4 params = bf(S, i, kRingParams);
    const d3 n = D(xyz(plane)), d = D(r.d);
    const double denom = dot(d, n);
    if (fabs(denom) < 1.0e-7) return miss;
    d3 oc;
    if (r.anchor == i) {
        oc = D(-r.o);
    } else if (r.anchor == kMiss) {
        oc = D(xyz(bf(S, i, kCenter))) + D(xyz(bf(S, i, kLow))) - D(r.o);
    } else {
        oc = (D(xyz(bf(S, i, kCenter))) - D(xyz(bf(S, r.anchor, kCenter)))) +
             (D(xyz(bf(S, i, kLow))) - D(xyz(bf(S, r.anchor, kLow)))) - D(r.o);
    }
    const double a = dot(d, d);
    const d3 perpendicular = cross(d, cross(d, oc)) * (1.0 / a);
    const double along = -dot(perpendicular, n) / denom;
    const double distance = dot(oc, d) / a + along;
    if (distance <= 0.0) return miss;
    const d3 point = perpendicular + d * along;
    const double radius = sqrt(dot(point, point)) / (double)b_radius(S, i);
    if (radius < (double)plane.w || radius > (double)params.x) return miss;
    return RingHit{(float)distance, i, F(point)};
}

// ring_hit (rings.wgsl:8-34), strict.
template <bool C, bool L, bool F>
__device__ __forceinline__ RingHit ring_hit(const Scene &S, Counter<C, L, F> K, const Ray &r, uint32_t i) {
    const RingHit miss{1.0e30f, kMiss, f3(0.0f, 0.0f, 0.0f)};
    const float4 plane = bf(S, i, kRingPlane);
    const float4 params = bf(S, i, kRingParams);
    if (params.x <= plane.w || params.y <= 0.0f) return miss;
    K.add(&Events::ring_tests);
    if constexpr (F) return ring_hit_fp64(S, r, i);
    const float3 n = xyz(plane);
    const float denom = dot_rn(r.d, n);
    if (fabsf(denom) < 1.0e-7f) return miss;
    const float3 oc = relative_center(S, r, i);
    const float a = dot_rn(r.d, r.d);
    // The ray's line passes farther from the centre than the annulus
    // reaches (|oc x d|^2 / a > (outer R)^2, with a 1e-3 margin far above
    // the rounding of either side): every point of the ray, the plane
    // crossing included, lies outside the annulus, so the exact test below
    // would miss.
    {
        const float3 pc = cross(oc, r.d);
        const float reach = params.x * b_radius(S, i);
        if (dot(pc, pc) > a * reach * reach * 1.001f) return miss;
    }
    const float3 perpendicular = div_rn(cross_rn(r.d, cross_rn(r.d, oc)), a);
    const float along = __fdiv_rn(-dot_rn(perpendicular, n), denom);
    const float distance = __fadd_rn(__fdiv_rn(dot_rn(oc, r.d), a), along);
    if (distance <= 0.0f) return miss;
    const float3 point = add_rn(perpendicular, mul_rn(r.d, along));
    const float radius = __fdiv_rn(length_rn(point), b_radius(S, i));
    if (radius < plane.w || radius > params.x) return miss;
    return RingHit{distance, i, point};
}

// closest_ring (rings.wgsl:36-45).
template <bool C, bool L, bool F>
__device__ __forceinline__ RingHit closest_ring(const Scene &S, Counter<C, L, F> K, const Ray &r, float limit,
                                                Cull cull = kTestAll) {
    RingHit best{limit, kMiss, f3(0.0f, 0.0f, 0.0f)};
    const uint32_t n = S.s->counts[0];
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (!cull.ring(i)) continue;
        const RingHit h = ring_hit(S, K, r, i);
        if (h.index != kMiss && h.t < best.t) best = h;
    }
    return best;
}

struct Optics {
    float3 color;
    float tau;
};

// The illustrative banded profile of rings.wgsl:56-79 (C/B/A rings,
// Cassini division, Encke and Keeler gaps). Out of line: its accurate sinf
// calls carry a large range-reduction path that the table and scalar
// profiles never need.
static __device__ __noinline__ Optics banded_optics(float x, float tau, float3 color) {
    const float broad = 0.5f + 0.5f * sinf(43.0f * x + 1.8f * sinf(17.0f * x));
    const float fine = 0.5f + 0.5f * sinf(1900.0f * x + 2.0f * sinf(311.0f * x));
    const float micro = 0.5f + 0.5f * sinf(6100.0f * x);
    float density = 0.12f;
    float3 tint = f3(0.70f, 0.68f, 0.65f);
    if (x >= 0.2792f && x < 0.6910f) {
        density = 1.25f + 1.1f * broad;
        tint = f3(1.0f, 1.0f, 1.0f);
    } else if (x >= 0.6910f && x < 0.7649f) {
        density = 0.025f;
        tint = f3(0.75f, 0.75f, 0.75f);
    } else if (x >= 0.7649f) {
        density = 0.48f + 0.22f * broad;
        tint = f3(0.92f, 0.94f, 0.98f);
    }
    density *= 0.65f + 0.45f * fine + 0.12f * micro;
    if (fabsf(x - 0.9487f) < 0.00262f || fabsf(x - 0.99565f) < 0.00034f) density = 0.0f;
    return Optics{color * tint * (0.94f + 0.06f * broad), tau * density};
}

// Normalised ring radius x of a planet-local point (rings.wgsl:52-53).
__device__ __forceinline__ float ring_x(const Scene &S, uint32_t i, float3 point) {
    const float inner = bf(S, i, kRingPlane).w;
    const float outer = bf(S, i, kRingParams).x;
    const float radius = __fdiv_rn(length_rn(point), b_radius(S, i));
    return __fdiv_rn(__fsub_rn(radius, inner), __fsub_rn(outer, inner));
}

// Table bin of x for a ring-table slot (extension).
__device__ __forceinline__ uint32_t ring_bin(float x, uint32_t bins) {
    const float fb = x * (float)bins;
    const uint32_t bin = fb <= 0.0f ? 0u : (uint32_t)fb;
    return bin > bins - 1u ? bins - 1u : bin;
}

// ring_optics (rings.wgsl:50-81) plus the tabulated profile extension.
__device__ __forceinline__ Optics ring_optics(const Scene &S, uint32_t i, float3 point) {
    const float4 params = bf(S, i, kRingParams);
    const float x = ring_x(S, i, point);
    const float tau = params.y;
    const float3 color = xyz(bf(S, i, kRingColor));
    if (params.w >= 0.5f) {
        const uint32_t slot = (uint32_t)params.w - 1u;
        const uint32_t bins = slot < SG_RING_TABLE_SLOTS ? S.p->bins[slot] : 0u;
        if (bins == 0u) return Optics{color, 0.0f};
        return Optics{color, tau * S.tables[slot * S.p->table_stride + ring_bin(x, bins)]};
    }
    if (params.z > 0.5f) return banded_optics(x, tau, color);
    return Optics{color, tau};
}

// exp(-tau / |mu|); mu uses the strict dot so the optical path tau/|mu|
// rounds exactly as in an IEEE evaluation of the WGSL.
__device__ __forceinline__ float ring_transmission_tau(float3 d, float3 pole, float tau) {
    const float mu = fmaxf(fabsf(dot_rn(d, pole)), 1.0e-7f);
    return expf(__fdiv_rn(-tau, mu));
}

// ring_transmission (rings.wgsl:83-86).
__device__ __forceinline__ float ring_transmission(const Scene &S, const Ray &r, const RingHit &h) {
    return ring_transmission_tau(r.d, xyz(bf(S, h.index, kRingPlane)), ring_optics(S, h.index, h.p).tau);
}

// The ring crossings behind a visibility, for the adjoint: body and
// planet-local point of each (the first kMaxRecordedCrossings).
constexpr int kMaxRecordedCrossings = 2;
struct Crossings {
    uint32_t n;
    uint32_t body[kMaxRecordedCrossings];
    float3 point[kMaxRecordedCrossings];
};

// light_visibility (rings.wgsl:90-115): distance to the light, any-hit over
// the other spheres (ties broken by index), then ring transmissions before
// the light. With a Crossings record it also lists the ring crossings.
template <bool C, bool L, bool F>
__device__ __forceinline__ float visibility_core(const Scene &S, Counter<C, L, F> K, const Ray &r, uint32_t light,
                                                 Crossings *record) {
    K.add(&Events::shadow_rays);
    float delta;
    const float surface = sphere_distance(S, K, r, light, b_radius(S, light), delta);
    if (surface >= 1.0e30f) return 0.0f;
    const float host = S.s->g.ground_north[3];
    const uint32_t n = S.s->counts[0];
    if (host == (float)(light + 1u) && closest_hit(S, K, r).index != light) return 0.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (i == light || host == (float)(i + 1u)) continue;
        const float t = sphere_distance(S, K, r, i, b_radius(S, i), delta);
        if (t < 1.0e30f && (t < surface || (t == surface && i < light))) return 0.0f;
    }
    if constexpr (L) {
        if (host != 0.0f) {
            const LandHit local = landscape_query(S, K, r, surface, true);
            if (local.index != kMiss && local.t < surface) return 0.0f;
        }
    }
    float transmission = 1.0f;
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        const RingHit h = ring_hit(S, K, r, i);
        if (h.index != kMiss && h.t < surface) {
            transmission *= ring_transmission(S, r, h);
            if (record) {
                if (record->n < (uint32_t)kMaxRecordedCrossings) {
                    record->body[record->n] = i;
                    record->point[record->n] = h.p;
                }
                record->n += 1u;
            }
        }
    }
    return transmission;
}

template <bool C, bool L, bool F>
static __device__ SG_HELPER float light_visibility(Scene S, Counter<C, L, F> K, Ray r, uint32_t light) {
    return visibility_core(S, K, r, light, nullptr);
}

// one_minus_exp (rings.wgsl:143-145).
__device__ __forceinline__ float one_minus_exp(float x) {
    return x < 1.0e-3f ? x * (1.0f - 0.5f * x) : 1.0f - expf(-x);
}

// ring_bsdf (rings.wgsl:151-166): exact single scattering in a finite slab.
static __device__ SG_HELPER float3 ring_bsdf(Optics o, float outgoing, float incoming) {
    const float mo = fmaxf(fabsf(outgoing), 1.0e-7f);
    const float mi = fmaxf(fabsf(incoming), 1.0e-7f);
    const float a = o.tau / mo;
    const float b = o.tau / mi;
    if (outgoing * incoming < 0.0f) {
        const float delta = fabsf(a - b);
        const float integral =
            delta < 1.0e-3f ? 1.0f - 0.5f * delta : one_minus_exp(delta) / fmaxf(delta, 1.0e-20f);
        const float factor = o.tau / (mo * mi) * expf(-fminf(a, b)) * integral;
        return o.color * (factor / (4.0f * kPi));
    }
    const float factor = one_minus_exp(a + b) / (mo + mi);
    return o.color * (factor / (4.0f * kPi));
}

// ring_origin (rings.wgsl:168-175): reproject onto the plane, then offset
// by 2e-6 planet radii towards the outgoing side.
__device__ __forceinline__ Ray ring_origin(const Scene &S, uint32_t index, float3 point, float3 direction) {
    const float3 n = xyz(bf(S, index, kRingPlane));
    const float sign = dot(direction, n) >= 0.0f ? 1.0f : -1.0f;
    const float3 p = point - n * dot(point, n);
    return Ray{p + n * (sign * b_radius(S, index) * 2.0e-6f), direction, index};
}

// ring_area (pathtrace.wgsl:1237-1241).
__device__ __forceinline__ float ring_area(const Scene &S, uint32_t i) {
    const float r = b_radius(S, i);
    const float outer = bf(S, i, kRingParams).x;
    const float inner = bf(S, i, kRingPlane).w;
    return kPi * r * r * (outer * outer - inner * inner);
}

struct Shine {
    float3 radiance;
    uint32_t rng;
};

// The ring point ringshine samples (pathtrace.wgsl:1252-1280) and the
// per-point factors its light loop needs; `valid` false when the point
// contributes nothing.
struct ShinePoint {
    float3 point;
    Optics optics;
    float mu_out;
    float scale;  // cos_surface * weight / (pi * pdf)
    uint32_t rng;
    bool valid;
};

template <bool C, bool L, bool F>
__device__ __forceinline__ ShinePoint shine_point(const Scene &S, Counter<C, L, F> K, uint32_t index, float3 origin,
                                                  float3 normal, bool last_vertex, uint32_t rng) {
    ShinePoint out;
    out.valid = false;
    const float3 n = xyz(bf(S, index, kRingPlane));
    const float inner = bf(S, index, kRingPlane).w;
    const float outer = bf(S, index, kRingParams).x;
    const float radius = sqrtf(mixf(inner * inner, outer * outer, rnd(K, rng))) * b_radius(S, index);
    float sp, cp;
    sincos_turn(rnd(K, rng), &sp, &cp);
    out.rng = rng;
    const float3 point = basis_direction(n, cp, sp, 0.0f) * radius;
    const float3 offset = point - origin;
    const float distance2 = dot(offset, offset);
    const float distance = sqrtf(distance2);
    const float3 direction = offset / distance;
    const float cos_surface = dot(normal, direction);
    const float cos_ring = fabsf(dot(direction, n));
    if (cos_surface <= 0.0f || cos_ring < 1.0e-6f) return out;
    float delta;
    const float blocker = sphere_distance(S, K, Ray{origin, direction, index}, index, b_radius(S, index), delta);
    if (blocker < distance) return out;
    out.optics = ring_optics(S, index, point);
    if (out.optics.tau == 0.0f) return out;
    out.point = point;
    out.mu_out = dot(-direction, n);
    const float pdf = distance2 / (ring_area(S, index) * cos_ring);
    const float weight = last_vertex ? 1.0f : power_weight(pdf, cos_surface / kPi);
    out.scale = cos_surface * weight / (kPi * pdf);
    out.valid = true;
    return out;
}

// ringshine (pathtrace.wgsl:1248-1296): NEE of a planet's own sunlit ring.
template <bool C, bool L, bool F>
static __device__ SG_HELPER Shine ringshine(Scene S, Counter<C, L, F> K, uint32_t index, float3 origin, float3 normal,
                                        bool last_vertex, uint32_t rng) {
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    if (!has_ring(S, index)) return Shine{zero, rng};
    const ShinePoint sp = shine_point(S, K, index, origin, normal, last_vertex, rng);
    rng = sp.rng;
    if (!sp.valid) return Shine{zero, rng};
    const float3 n = xyz(bf(S, index, kRingPlane));
    float3 shine = zero;
    const uint32_t count = light_count(S.s);
#pragma unroll 1
    for (uint32_t slot = 0; slot < count; ++slot) {
        const uint32_t i = light_index(S.s, slot);
        const float4 material = bf(S, i, kMaterial);
        if (material.w < 0.5f) continue;
        const LightSample light = sample_light(S, K, Ray{sp.point, n, index}, i, rng);
        rng = light.rng;
        const float mu_in = dot(light.d, n);
        const float visibility = light_visibility(S, K, ring_origin(S, index, sp.point, light.d), i);
        shine = shine + ring_bsdf(sp.optics, sp.mu_out, mu_in) * xyz(material) * (fabsf(mu_in) * visibility / light.pdf);
    }
    return Shine{shine * sp.scale, rng};
}

// ---------------------------------------------------------------------------
// Camera-only sky backdrop (pathtrace.wgsl:268-334): catalogue star discs and
// the Milky Way panorama, seen along unscattered camera paths.
// ---------------------------------------------------------------------------
constexpr uint32_t kSkyGridW = 256, kSkyGridH = 128;

// world_direction (pathtrace.wgsl:268-271).
__device__ __forceinline__ float3 world_direction(const sg_settings *s, float3 d) {
    const float3 r = f3(s->g.cam_right[0], s->g.cam_right[1], s->g.cam_right[2]);
    const float3 u = f3(s->g.cam_up[0], s->g.cam_up[1], s->g.cam_up[2]);
    const float3 f = f3(s->g.cam_forward[0], s->g.cam_forward[1], s->g.cam_forward[2]);
    return normalize(r * d.x + u * d.y - f * d.z);
}

// inside_star_dot (pathtrace.wgsl:118-128): within kStarDotPixels of the
// star's projected centre.
__device__ __forceinline__ bool inside_star_dot(const sg_settings *s, float3 view, float3 star) {
    const float3 r = f3(s->g.cam_right[0], s->g.cam_right[1], s->g.cam_right[2]);
    const float3 u = f3(s->g.cam_up[0], s->g.cam_up[1], s->g.cam_up[2]);
    const float3 f = f3(s->g.cam_forward[0], s->g.cam_forward[1], s->g.cam_forward[2]);
    const float3 sv = f3(dot(star, r), dot(star, u), -dot(star, f));
    if (sv.z >= 0.0f) return false;
    const float dx = view.x / -view.z - sv.x / -sv.z, dy = view.y / -view.z - sv.y / -sv.z;
    const float scale = s->g.viewport[1] / (2.0f * s->g.cam_forward[3]);
    const float px = dx * scale, py = dy * scale;
    return px * px + py * py <= kStarDotPixels * kStarDotPixels;
}

// environment (pathtrace.wgsl:273-300) of a primary ray: the catalogue
// discs listed in the direction's grid cell.
static __device__ __noinline__ float3 environment(const TraceParams *P, float3 view) {
    float3 light = f3(0.0f, 0.0f, 0.0f);
    if (P->catalogue_n == 0u) return light;
    const float3 dir = world_direction(&P->s, view);
    const float phi = atan2f(dir.y, dir.x) + kPi;
    const float theta = acosf(clampf(dir.z, -1.0f, 1.0f));
    const uint32_t x = min((uint32_t)(phi * (256.0f / kTau)), kSkyGridW - 1u);
    const uint32_t y = min((uint32_t)(theta * (128.0f / kPi)), kSkyGridH - 1u);
    const uint32_t cell = y * kSkyGridW + x;
    const uint32_t *cells = P->sky_cells;
    for (uint32_t j = cells[cell]; j < cells[cell + 1u]; ++j) {
        const uint32_t k = cells[kSkyGridW * kSkyGridH + 1u + j];
        const float4 sd = P->catalogue[2u * k];
        const float3 sdir = xyz(sd);
        const float3 perp = cross(dir, sdir);
        if (dot(dir, sdir) > 0.0f && dot(perp, perp) <= sd.w && inside_star_dot(&P->s, view, sdir))
            light = light + xyz(P->catalogue[2u * k + 1u]);
    }
    return light;
}

// milky_way_texel / milky_way (pathtrace.wgsl:302-334): the panorama in
// galactic coordinates (pole normalize(0.35, 0.82, 0.45), Duff basis),
// bilinear, times the backdrop brightness.
__device__ __forceinline__ float3 milky_way_texel(const TraceParams *P, int x, int y) {
    const int w = (int)P->s.background[1], h = (int)P->s.background[2];
    x = (x + w) % w;
    y = min(max(y, 0), h - 1);
    const uint32_t t = P->milky_way[(uint32_t)(y * w + x)];
    return f3((float)(t & 1023u), (float)((t >> 10) & 1023u), (float)((t >> 20) & 1023u)) / 1023.0f;
}
static __device__ __noinline__ float3 milky_way(const TraceParams *P, float3 view) {
    if (P->s.background[0] == 0.0f || !P->milky_way) return f3(0.0f, 0.0f, 0.0f);
    const float3 dir = world_direction(&P->s, view);
    const float3 pole = normalize(f3(0.35f, 0.82f, 0.45f));
    const float a = -1.0f / (1.0f + pole.z);
    const float3 right = f3(pole.x * pole.y * a, 1.0f + pole.y * pole.y * a, -pole.y);
    const float3 forward = cross(pole, right);
    const float longitude = atan2f(dot(dir, forward), dot(dir, right));
    const float u = 0.5f - longitude / kTau;
    const float v = acosf(clampf(dot(dir, pole), -1.0f, 1.0f)) / kPi;
    const float px = u * P->s.background[1] - 0.5f, py = v * P->s.background[2] - 0.5f;
    const float fx = floorf(px), fy = floorf(py);
    const int lx = (int)fx, ly = (int)fy;
    const float wx = px - fx, wy = py - fy;
    const float3 t00 = milky_way_texel(P, lx, ly), t10 = milky_way_texel(P, lx + 1, ly);
    const float3 t01 = milky_way_texel(P, lx, ly + 1), t11 = milky_way_texel(P, lx + 1, ly + 1);
    const float3 top = t00 * (1.0f - wx) + t10 * wx, bot = t01 * (1.0f - wx) + t11 * wx;
    return (top * (1.0f - wy) + bot * wy) * P->s.background[0];
}

// point_gain (pathtrace.wgsl:1341-1345).
__device__ __forceinline__ float point_gain(const sg_settings *s, float extent, float distance) {
    const float pixel = 2.0f * s->g.cam_forward[3] / fmaxf(s->g.viewport[1], 1.0f);
    const float pixels = 2.0f * extent / fmaxf(distance, 1.0e-30f) / pixel;
    return mixf(s->background[3], 1.0f, smoothstepf(1.0f, 3.0f, pixels));
}

struct DiscHit {
    Hit hit;
    float scale;
    uint32_t rng;
};

// point_disc_hit (pathtrace.wgsl:1308-1333): depth-0 camera rays see an
// unresolved body as a disc of at least a bright star's size.
template <bool C, bool L, bool F>
static __device__ SG_HELPER DiscHit point_disc_hit(Scene S, Counter<C, L, F> K, Ray r, Hit closest, uint32_t rng,
                                                   Cull cull = kTestAll) {
    const sg_settings *s = S.s;
    DiscHit out{closest, 1.0f, rng};
    float total = 0.0f;
    const float pixel = 2.0f * s->g.cam_forward[3] / fmaxf(s->g.viewport[1], 1.0f);
    const float angle = clampf(kPointDiscRadius, 0.7f * pixel, kStarDotPixels * pixel);
    const uint32_t host = (uint32_t)s->g.atmo_params[3] - 1u;
    const uint32_t n = s->counts[0];
#pragma unroll 1
    for (uint32_t i = 0; i < n; ++i) {
        if (i == host || s->g.ground_north[3] == (float)(i + 1u) || !cull.body(i)) continue;
        const float radius = b_radius(S, i);
        const float drawn = __fmul_rn(angle, length_rn(relative_center(S, r, i)));
        if (radius <= 0.0f || drawn <= radius) continue;
        float delta;
        const float t = sphere_distance(S, K, r, i, drawn, delta);
        if (t < closest.t) {
            const float ratio = (radius / drawn) * (radius / drawn);
            total += ratio;
            if (rnd(K, out.rng) * total < ratio) out.hit = Hit{t, i, delta, f3(0.0f, 0.0f, 0.0f)};
        }
    }
    if (total > 0.0f) out.scale = total;
    return out;
}

// ---------------------------------------------------------------------------
// Surface albedo, style 0 with optional value-noise mottle
// (pathtrace.wgsl:338-354, :377-389, :897-925).
// ---------------------------------------------------------------------------
// Value noise is strict: fract() of scaled coordinates amplifies any
// contraction difference into a different lattice hash, so the noise is
// evaluated exactly as an IEEE reading of the WGSL.
__device__ __forceinline__ float fractf(float x) { return __fsub_rn(x, floorf(x)); }
__device__ __forceinline__ float mix_rn(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}
__device__ __forceinline__ float hash31(float3 p) {
    float3 q = f3(fractf(__fmul_rn(p.x, 0.1031f)), fractf(__fmul_rn(p.y, 0.1030f)), fractf(__fmul_rn(p.z, 0.0973f)));
    const float d = dot_rn(q, f3(__fadd_rn(q.y, 33.33f), __fadd_rn(q.x, 33.33f), __fadd_rn(q.z, 33.33f)));
    q = f3(__fadd_rn(q.x, d), __fadd_rn(q.y, d), __fadd_rn(q.z, d));
    return fractf(__fmul_rn(__fadd_rn(q.x, q.y), q.z));
}
__device__ __forceinline__ float smooth_rn(float f) {
    return __fmul_rn(__fmul_rn(f, f), __fsub_rn(3.0f, __fmul_rn(2.0f, f)));
}
static __device__ __noinline__ float vnoise(float3 p) {
    const float3 i = f3(floorf(p.x), floorf(p.y), floorf(p.z));
    const float3 f = sub_rn(p, i);
    const float3 u = f3(smooth_rn(f.x), smooth_rn(f.y), smooth_rn(f.z));
    const float a = mix_rn(hash31(i), hash31(add_rn(i, f3(1, 0, 0))), u.x);
    const float b = mix_rn(hash31(add_rn(i, f3(0, 1, 0))), hash31(add_rn(i, f3(1, 1, 0))), u.x);
    const float c = mix_rn(hash31(add_rn(i, f3(0, 0, 1))), hash31(add_rn(i, f3(1, 0, 1))), u.x);
    const float d = mix_rn(hash31(add_rn(i, f3(0, 1, 1))), hash31(add_rn(i, f3(1, 1, 1))), u.x);
    return mix_rn(mix_rn(a, b, u.y), mix_rn(c, d, u.y), u.z);
}

// Mottle factor of surface_albedo (pathtrace.wgsl:912-923), out of line:
// five octaves of value noise that the constant-albedo path never runs.
static __device__ __noinline__ float mottle(float3 axis_x, float4 axis_y, float strength, float3 normal) {
    const float3 y = xyz(axis_y);
    const float3 local = f3(dot_rn(normal, axis_x), dot_rn(normal, y), dot_rn(normal, cross_rn(axis_x, y)));
    const float seed = axis_y.w;
    const float3 off =
        f3(hash31(f3(seed, 1.0f, 7.0f)), hash31(f3(3.0f, seed, 5.0f)), hash31(f3(9.0f, 2.0f, seed))) * 512.0f;
    float3 p = add_rn(mul_rn(local, 2.4f), off);
    float amplitude = 0.5f, noise = 0.0f;
    for (int octave = 0; octave < 5; ++octave) {
        noise = __fadd_rn(noise, __fmul_rn(amplitude, vnoise(p)));
        p = mul_rn(p, 2.07f);
        amplitude *= 0.5f;
    }
    return mix_rn(1.0f, __fadd_rn(0.68f, __fmul_rn(0.64f, noise)), strength);
}

}  // namespace sg

#include "sg_surface.cuh"
