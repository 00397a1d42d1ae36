/*
 * oracle.c — CPU restatement of stargaze's progressive path-tracing
 * integrator. TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels,
 * never part of the product path. See oracle.h for the parity pin.
 *
 * Every function names the WGSL it restates. Expression order follows the
 * WGSL source; the file must be compiled with -ffp-contract=off and without
 * -ffast-math so that f32 + - * / sqrt round exactly as written.
 *
 * Scope: the integrator of pathtrace.wgsl (sample loop, spheres, rings,
 * stellar NEE with MIS, ringshine, point discs, Russian roulette,
 * running-mean accumulation) and rings.wgsl; the host atmosphere with its
 * camera-air pass and surface sky cache; the catalogue and Milky Way
 * backdrop; procedural surface styles 1-6; the local landscape of
 * ground.wgsl, terrain.wgsl, volcano.wgsl and forest.wgsl (themes 0-5,
 * props, vegetation); the guided ground sampler (src/guided_ground.rs).
 * Where the WGSL hashes coordinates derived from transcendental functions
 * (surface styles, themes 3-5, vegetation), those functions are evaluated
 * in double and rounded to f32, as the CUDA path does.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>

/* The arithmetic type: f32, the reference's (the default build), or f64
 * when built with -DORACLE_F64 (liboracle_f64.so: converged reference images
 * free of f32 rounding). Buffers shared with the caller stay float either
 * way. */
#ifdef ORACLE_F64
typedef double real;
#define r_acos acos
#define r_atan2 atan2
#define r_ceil ceil
#define r_cos cos
#define r_exp exp
#define r_fabs fabs
#define r_floor floor
#define r_fmod fmod
#define r_pow pow
#define r_rint rint
#define r_sin sin
#define r_sqrt sqrt
#else
typedef float real;
#define r_acos acosf
#define r_atan2 atan2f
#define r_ceil ceilf
#define r_cos cosf
#define r_exp expf
#define r_fabs fabsf
#define r_floor floorf
#define r_fmod fmodf
#define r_pow powf
#define r_rint rintf
#define r_sin sinf
#define r_sqrt sqrtf
#endif
#endif

#define PI_F 3.141592653589793f
#define TAU_F 6.283185307179586f
#define MISS SG_MISS
#define LOCAL_BASE SG_LOCAL_BASE
#define STAR_DOT_PIXELS 3.0f
#define POINT_DISC_RADIUS 0.00136f
#define RING_INDIRECT_CAP 0.003f

/* ---------------------------------------------------------------- */
/* Small vector algebra (WGSL vec3<f32> semantics, fixed order).     */
/* ---------------------------------------------------------------- */
typedef struct { real x, y, z; } v3;

static inline v3 V(real x, real y, real z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 vmul(v3 a, real s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vmulv(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vdivs(v3 a, real s) { return V(a.x / s, a.y / s, a.z / s); }
static inline real vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline real vlength(v3 a) { return r_sqrt(vdot(a, a)); }
static inline v3 vnormalize(v3 a) { real inv = 1.0f / r_sqrt(vdot(a, a)); return vmul(a, inv); }
static inline real minf_(real a, real b) { return a < b ? a : b; }
static inline real maxf_(real a, real b) { return a > b ? a : b; }
static inline real clampf_(real x, real lo, real hi) { return minf_(maxf_(x, lo), hi); }
static inline real mixf(real a, real b, real t) { return a * (1.0f - t) + b * t; }
static inline real fractf(real x) { return x - r_floor(x); }
static inline real smoothstepf(real e0, real e1, real x) {
    real t = clampf_((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
static inline real lum(v3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

/* ---------------------------------------------------------------- */
/* Scene access                                                      */
/* ---------------------------------------------------------------- */
/* What integrate_camera_air leaves for trace (pathtrace.wgsl:1629-1643). */
typedef struct { real radiance[3]; uint32_t rng; } camera_air_t;

typedef struct {
    const sg_settings *s;
    const sg_sphere *b;
    const oracle_tables *t;
    oracle_events *ev;
    const real *sky;          /* surface sky cache, 128 x float4 (air frames) */
    const camera_air_t *air;   /* this sample's camera air (air frames) */
} scene;

typedef struct { v3 offset; v3 dir; uint32_t anchor; } ray_t;   /* pathtrace.wgsl:70-76 */
typedef struct { real distance; uint32_t index; v3 normal; } hit_t; /* :77-81 */
typedef struct { v3 dir; real pdf; } light_sample; /* :82-85 */
typedef struct { real distance; uint32_t index; v3 point; } ring_hit_t; /* rings.wgsl:2-6 */

static inline v3 b_center(const scene *S, uint32_t i) { return V(S->b[i].center[0], S->b[i].center[1], S->b[i].center[2]); }
static inline v3 b_low(const scene *S, uint32_t i) { return V(S->b[i].center_low[0], S->b[i].center_low[1], S->b[i].center_low[2]); }
static inline real b_radius(const scene *S, uint32_t i) { return S->b[i].radius; }
static inline v3 b_color(const scene *S, uint32_t i) { return V(S->b[i].color[0], S->b[i].color[1], S->b[i].color[2]); }
static inline real b_emissive(const scene *S, uint32_t i) { return S->b[i].emissive; }
static inline v3 b_pole(const scene *S, uint32_t i) { return V(S->b[i].ring_plane[0], S->b[i].ring_plane[1], S->b[i].ring_plane[2]); }
#define EV(field) do { if (S->ev) S->ev->field++; } while (0)

/* hash, random: pathtrace.wgsl:87-98 */
static inline uint32_t hash_u32(uint32_t value) {
    uint32_t x = value;
    x = (x ^ (x >> 16)) * 0x7feb352du;
    x = (x ^ (x >> 15)) * 0x846ca68bu;
    return x ^ (x >> 16);
}
static inline real rnd(const scene *S, uint32_t *state) {
    EV(rng_draws);
    *state = *state * 747796405u + 2891336453u;
    uint32_t word = ((*state >> ((*state >> 28) + 4u)) ^ *state) * 277803737u;
    return (real)(((word >> 22) ^ word) >> 8) * (1.0f / 16777216.0f);
}

/* relative_center: pathtrace.wgsl:100-113 */
static v3 relative_center(const scene *S, ray_t ray, uint32_t index) {
    if (ray.anchor == index) return vneg(ray.offset);
    if (ray.anchor == MISS) return vadd(b_center(S, index), vsub(b_low(S, index), ray.offset));
    return vadd(vsub(b_center(S, index), b_center(S, ray.anchor)),
                vsub(vsub(b_low(S, index), b_low(S, ray.anchor)), ray.offset));
}

static inline hit_t miss_hit(void) { hit_t h = {1.0e30f, MISS, {0, 0, 0}}; return h; }

/* sphere_hit_radius: pathtrace.wgsl:134-171 */
static hit_t sphere_hit_radius(const scene *S, ray_t ray, uint32_t index, real radius) {
    EV(sphere_tests);
    v3 oc = relative_center(S, ray, index);
    real a = vdot(ray.dir, ray.dir);
    real b = vdot(oc, ray.dir);
    v3 pc = vcross(oc, ray.dir);
    real h = a * radius * radius - vdot(pc, pc);
    if (h < 0.0f) return miss_hit();
    real root = r_sqrt(h);
    real q = b + (b >= 0.0f ? root : -root);
    if (q == 0.0f) return miss_hit();
    real c = vdot(oc, oc) - radius * radius;
    real near_ = (b < 0.0f) ? q / a : c / q;
    real far_ = (b < 0.0f) ? c / q : q / a;
    real distance = near_;
    real delta = -root / a;
    if (distance <= 0.0f) { distance = far_; delta = root / a; }
    if (distance <= 0.0f) return miss_hit();
    EV(sphere_hits);
    v3 perpendicular = vdivs(vcross(ray.dir, pc), a);
    hit_t hit;
    hit.distance = distance;
    hit.index = index;
    hit.normal = vnormalize(vadd(vneg(perpendicular), vmul(ray.dir, delta)));
    return hit;
}
static inline hit_t sphere_hit(const scene *S, ray_t ray, uint32_t index) {
    return sphere_hit_radius(S, ray, index, b_radius(S, index));
}

/* landscape_query: ground.wgsl:123-242 (defined with the landscape code). */
static hit_t landscape_query(const scene *S, ray_t ray, real limit, int occlusion);

/* closest_hit: pathtrace.wgsl:173-185 */
static hit_t closest_hit(const scene *S, ray_t ray) {
    hit_t closest = miss_hit();
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (S->s->g.ground_north[3] == (real)(i + 1u)) continue;
        hit_t hit = sphere_hit(S, ray, i);
        if (hit.distance < closest.distance) closest = hit;
    }
    hit_t local = landscape_query(S, ray, 1.0e30f, 0);
    if (local.distance < closest.distance) closest = local;
    return closest;
}

/* basis_direction: pathtrace.wgsl:187-194 */
static v3 basis_direction(v3 axis, real x, real y, real z) {
    v3 helper = V(0.0f, 0.0f, 1.0f);
    if (r_fabs(axis.z) > 0.9f) helper = V(0.0f, 1.0f, 0.0f);
    v3 tangent = vnormalize(vcross(helper, axis));
    return vnormalize(vadd(vadd(vmul(tangent, x), vmul(vcross(axis, tangent), y)), vmul(axis, z)));
}

/* cone_width: pathtrace.wgsl:197-202 */
static real cone_width(const scene *S, ray_t ray, uint32_t index) {
    v3 oc = relative_center(S, ray, index);
    real r = b_radius(S, index);
    real sin2 = clampf_(r * r / vdot(oc, oc), 1.0e-20f, 1.0f);
    return sin2 / (1.0f + r_sqrt(1.0f - sin2));
}

/* light_count, light_index: pathtrace.wgsl:205-211 */
static inline uint32_t light_count(const scene *S) {
    return S->s->lights[3] <= 3u ? S->s->lights[3] : S->s->counts[0];
}
static inline uint32_t light_index(const scene *S, uint32_t slot) {
    if (S->s->lights[3] <= 3u) return S->s->lights[slot];
    return slot;
}

/* sample_light_stratum / sample_light: pathtrace.wgsl:214-234 */
static light_sample sample_light_stratum(const scene *S, ray_t ray, uint32_t index,
                                         uint32_t stratum, uint32_t count, uint32_t *rng) {
    EV(light_samples);
    v3 axis = vnormalize(relative_center(S, ray, index));
    real width = cone_width(S, ray, index);
    real radial = rnd(S, rng);
    real azimuth = rnd(S, rng);
    if (count == 4u) {
        radial = ((real)(stratum & 1u) + radial) * 0.5f;
        azimuth = ((real)(stratum >> 1u) + azimuth) * 0.5f;
    }
    real one_minus_cos = radial * width;
    real sin_theta = r_sqrt(one_minus_cos * (2.0f - one_minus_cos));
    real phi = TAU_F * azimuth;
    light_sample ls;
    ls.dir = basis_direction(axis, sin_theta * r_cos(phi), sin_theta * r_sin(phi), 1.0f - one_minus_cos);
    ls.pdf = 1.0f / (TAU_F * width);
    return ls;
}
static inline light_sample sample_light(const scene *S, ray_t ray, uint32_t index, uint32_t *rng) {
    return sample_light_stratum(S, ray, index, 0u, 1u, rng);
}

/* power_weight: pathtrace.wgsl:264-267 */
static inline real power_weight(real a, real b) {
    real ratio = b / maxf_(a, 1.0e-30f);
    return 1.0f / (1.0f + ratio * ratio);
}

/* ---------------------------------------------------------------- */
/* Rings: rings.wgsl                                                 */
/* ---------------------------------------------------------------- */
static inline ring_hit_t ring_miss(real limit) { ring_hit_t r = {limit, MISS, {0, 0, 0}}; return r; }

/* ring_hit: rings.wgsl:8-34 */
static ring_hit_t ring_hit(const scene *S, ray_t ray, uint32_t index) {
    const sg_sphere *body = &S->b[index];
    if (body->ring_params[0] <= body->ring_plane[3] || body->ring_params[1] <= 0.0f) return ring_miss(1.0e30f);
    EV(ring_tests);
    v3 n = b_pole(S, index);
    real denom = vdot(ray.dir, n);
    if (r_fabs(denom) < 1.0e-7f) return ring_miss(1.0e30f);
    v3 oc = relative_center(S, ray, index);
    real a = vdot(ray.dir, ray.dir);
    v3 perpendicular = vdivs(vcross(ray.dir, vcross(ray.dir, oc)), a);
    real along = -vdot(perpendicular, n) / denom;
    real distance = vdot(oc, ray.dir) / a + along;
    if (distance <= 0.0f) return ring_miss(1.0e30f);
    v3 point = vadd(perpendicular, vmul(ray.dir, along));
    real radius = vlength(point) / body->radius;
    if (radius < body->ring_plane[3] || radius > body->ring_params[0]) return ring_miss(1.0e30f);
    ring_hit_t r = {distance, index, point};
    return r;
}

/* closest_ring: rings.wgsl:36-45 */
static ring_hit_t closest_ring(const scene *S, ray_t ray, real limit) {
    ring_hit_t closest = ring_miss(limit);
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS && hit.distance < closest.distance) closest = hit;
    }
    return closest;
}

typedef struct { v3 color; real tau; } optics_t;

/* ring_optics: rings.wgsl:50-81, plus the tabulated-profile extension
 * (ring_params.w = slot + 1): tau = ring_params.y * table[bin(x)]. */
static optics_t ring_optics(const scene *S, uint32_t index, v3 point) {
    const sg_sphere *body = &S->b[index];
    real radius = vlength(point) / body->radius;
    real x = (radius - body->ring_plane[3]) / (body->ring_params[0] - body->ring_plane[3]);
    real tau = body->ring_params[1];
    v3 color = V(body->ring_color[0], body->ring_color[1], body->ring_color[2]);
    if (body->ring_params[3] >= 0.5f) {
        uint32_t slot = (uint32_t)body->ring_params[3] - 1u;
        const float *table = (S->t && slot < SG_RING_TABLE_SLOTS) ? S->t->ring_tau[slot] : NULL;
        uint32_t bins = table ? S->t->ring_bins[slot] : 0u;
        if (bins > 0u) {
            real fb = x * (real)bins;
            uint32_t bin = fb <= 0.0f ? 0u : (uint32_t)fb;
            if (bin > bins - 1u) bin = bins - 1u;
            tau *= table[bin];
        } else {
            tau = 0.0f;
        }
    } else if (body->ring_params[2] > 0.5f) {
        real broad = 0.5f + 0.5f * r_sin(43.0f * x + 1.8f * r_sin(17.0f * x));
        real fine = 0.5f + 0.5f * r_sin(1900.0f * x + 2.0f * r_sin(311.0f * x));
        real micro = 0.5f + 0.5f * r_sin(6100.0f * x);
        real density = 0.12f;
        v3 tint = V(0.70f, 0.68f, 0.65f);
        if (x >= 0.2792f && x < 0.6910f) {
            density = 1.25f + 1.1f * broad;
            tint = V(1.0f, 1.0f, 1.0f);
        } else if (x >= 0.6910f && x < 0.7649f) {
            density = 0.025f;
            tint = V(0.75f, 0.75f, 0.75f);
        } else if (x >= 0.7649f) {
            density = 0.48f + 0.22f * broad;
            tint = V(0.92f, 0.94f, 0.98f);
        }
        density *= 0.65f + 0.45f * fine + 0.12f * micro;
        if (r_fabs(x - 0.9487f) < 0.00262f || r_fabs(x - 0.99565f) < 0.00034f) density = 0.0f;
        tau *= density;
        color = vmul(vmulv(color, tint), 0.94f + 0.06f * broad);
    }
    optics_t o = {color, tau};
    return o;
}

/* ring_transmission: rings.wgsl:83-86 */
static real ring_transmission(const scene *S, ray_t ray, ring_hit_t hit) {
    real mu = maxf_(r_fabs(vdot(ray.dir, b_pole(S, hit.index))), 1.0e-7f);
    return r_exp(-ring_optics(S, hit.index, hit.point).tau / mu);
}

/* light_visibility: rings.wgsl:90-115 */
static real light_visibility(const scene *S, ray_t ray, uint32_t light) {
    EV(shadow_rays);
    hit_t surface = sphere_hit(S, ray, light);
    if (surface.index == MISS) return 0.0f;
    if (S->s->g.ground_north[3] == (real)(light + 1u) && closest_hit(S, ray).index != light) return 0.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (i == light || S->s->g.ground_north[3] == (real)(i + 1u)) continue;
        hit_t hit = sphere_hit(S, ray, i);
        if (hit.index != MISS && (hit.distance < surface.distance ||
                                  (hit.distance == surface.distance && i < light)))
            return 0.0f;
    }
    hit_t local = landscape_query(S, ray, surface.distance, 1);
    if (local.index != MISS && local.distance < surface.distance) return 0.0f;
    real transmission = 1.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS && hit.distance < surface.distance) transmission *= ring_transmission(S, ray, hit);
    }
    return transmission;
}

/* one_minus_exp: rings.wgsl:143-145 */
static inline real one_minus_exp(real x) {
    return x < 1.0e-3f ? x * (1.0f - 0.5f * x) : 1.0f - r_exp(-x);
}

/* ring_bsdf: rings.wgsl:151-166; ring_factor is its scalar part. */
static real ring_factor(real tau, real outgoing, real incoming) {
    real mo = maxf_(r_fabs(outgoing), 1.0e-7f);
    real mi = maxf_(r_fabs(incoming), 1.0e-7f);
    real a = tau / mo;
    real b = tau / mi;
    if (outgoing * incoming < 0.0f) {
        real delta = r_fabs(a - b);
        real integral = delta < 1.0e-3f ? 1.0f - 0.5f * delta
                                         : one_minus_exp(delta) / maxf_(delta, 1.0e-20f);
        return tau / (mo * mi) * r_exp(-minf_(a, b)) * integral;
    }
    return one_minus_exp(a + b) / (mo + mi);
}
static v3 ring_bsdf(optics_t optics, real outgoing, real incoming) {
    return vmul(optics.color, ring_factor(optics.tau, outgoing, incoming) / (4.0f * PI_F));
}

/* ---------------------------------------------------------------- */
/* Forward-mode tangents of the detached estimator (adjoint check).   */
/* A direction D assigns a tangent to every material parameter; the   */
/* functions below return d(value) along D with geometry and every    */
/* sampling decision held fixed.                                      */
/* ---------------------------------------------------------------- */
static inline v3 dir_body_color(const oracle_direction *D, uint32_t i) {
    if (!D || !D->body_color) return V(0, 0, 0);
    return V(D->body_color[3 * i], D->body_color[3 * i + 1], D->body_color[3 * i + 2]);
}

/* Tangent of ring_optics at a ring point. */
static optics_t ring_optics_dot(const scene *S, const oracle_direction *D, uint32_t index, v3 point) {
    const sg_sphere *body = &S->b[index];
    optics_t d = {V(0, 0, 0), 0.0f};
    if (!D) return d;
    v3 dcolor = D->ring_albedo ? V(D->ring_albedo[3 * index], D->ring_albedo[3 * index + 1], D->ring_albedo[3 * index + 2])
                               : V(0, 0, 0);
    real radius = vlength(point) / body->radius;
    real x = (radius - body->ring_plane[3]) / (body->ring_params[0] - body->ring_plane[3]);
    if (body->ring_params[3] >= 0.5f) {
        uint32_t slot = (uint32_t)body->ring_params[3] - 1u;
        uint32_t bins = (S->t && slot < SG_RING_TABLE_SLOTS && S->t->ring_tau[slot]) ? S->t->ring_bins[slot] : 0u;
        if (bins > 0u) {
            real fb = x * (real)bins;
            uint32_t bin = fb <= 0.0f ? 0u : (uint32_t)fb;
            if (bin > bins - 1u) bin = bins - 1u;
            if (D->ring_tau[slot]) d.tau = body->ring_params[1] * D->ring_tau[slot][bin];
        }
        d.color = dcolor;
    } else if (body->ring_params[2] > 0.5f) {
        real broad = 0.5f + 0.5f * r_sin(43.0f * x + 1.8f * r_sin(17.0f * x));
        v3 tint = V(0.70f, 0.68f, 0.65f);
        if (x >= 0.2792f && x < 0.6910f) tint = V(1.0f, 1.0f, 1.0f);
        else if (x >= 0.6910f && x < 0.7649f) tint = V(0.75f, 0.75f, 0.75f);
        else if (x >= 0.7649f) tint = V(0.92f, 0.94f, 0.98f);
        d.color = vmul(vmulv(dcolor, tint), 0.94f + 0.06f * broad);
    } else {
        d.color = dcolor;
    }
    return d;
}

/* d factor / d tau of ring_bsdf, differentiating the same piecewise forms
 * (one_minus_exp's series below 1e-3, the integral's series below 1e-3). */
static real ring_factor_dtau(real tau, real outgoing, real incoming) {
    real mo = maxf_(r_fabs(outgoing), 1.0e-7f);
    real mi = maxf_(r_fabs(incoming), 1.0e-7f);
    if (outgoing * incoming < 0.0f) {
        real a = tau / mo, b = tau / mi;
        real delta = r_fabs(a - b);
        real k = r_fabs(1.0f / mo - 1.0f / mi);
        real m = minf_(1.0f / mo, 1.0f / mi);
        real integral, dintegral; /* value and d/d delta */
        if (delta < 1.0e-3f) {
            integral = 1.0f - 0.5f * delta;
            dintegral = -0.5f;
        } else {
            double dd = (double)delta, e = exp(-dd);
            integral = one_minus_exp(delta) / maxf_(delta, 1.0e-20f);
            dintegral = (real)((e * dd - (1.0 - e)) / (dd * dd));
        }
        real g = r_exp(-minf_(a, b));
        /* factor = tau / (mo mi) * g * integral */
        return (g * integral - tau * m * g * integral + tau * g * dintegral * k) / (mo * mi);
    }
    real k = 1.0f / mo + 1.0f / mi;
    real x = tau / mo + tau / mi;
    real dome = x < 1.0e-3f ? 1.0f - x : r_exp(-x);
    return k * dome / (mo + mi);
}

/* Tangent of ring_bsdf(optics, outgoing, incoming). */
static v3 ring_bsdf_dot(optics_t optics, optics_t doptics, real outgoing, real incoming) {
    real factor = ring_factor(optics.tau, outgoing, incoming);
    real dfactor = doptics.tau != 0.0f ? ring_factor_dtau(optics.tau, outgoing, incoming) * doptics.tau : 0.0f;
    return vadd(vmul(doptics.color, factor / (4.0f * PI_F)), vmul(optics.color, dfactor / (4.0f * PI_F)));
}

/* Tangent of light_visibility: the transmissions of the ring crossings
 * before the light (rings.wgsl:107-114), given the visibility `vis`. */
static real light_visibility_dot(const scene *S, const oracle_direction *D, ray_t ray, uint32_t light, real vis) {
    if (!D || vis <= 0.0f) return 0.0f;
    hit_t surface = sphere_hit(S, ray, light);
    real sum = 0.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index == MISS || !(hit.distance < surface.distance)) continue;
        real mu = maxf_(r_fabs(vdot(ray.dir, b_pole(S, i))), 1.0e-7f);
        sum += -ring_optics_dot(S, D, i, hit.point).tau / mu;
    }
    return vis * sum;
}

/* ring_origin: rings.wgsl:168-175 */
static ray_t ring_origin(const scene *S, ring_hit_t hit, v3 direction) {
    v3 n = b_pole(S, hit.index);
    real sign = vdot(direction, n) >= 0.0f ? 1.0f : -1.0f;
    v3 point = vsub(hit.point, vmul(n, vdot(hit.point, n)));
    ray_t r;
    r.offset = vadd(point, vmul(n, sign * b_radius(S, hit.index) * 2.0e-6f));
    r.dir = direction;
    r.anchor = hit.index;
    return r;
}

/* ring_area: pathtrace.wgsl:1237-1241 */
static real ring_area(const scene *S, uint32_t index) {
    const sg_sphere *body = &S->b[index];
    real r = body->radius;
    return PI_F * r * r * (body->ring_params[0] * body->ring_params[0] - body->ring_plane[3] * body->ring_plane[3]);
}

/* ringshine: pathtrace.wgsl:1248-1296. With a direction D, *dshine
 * receives the tangent of the result. */
static v3 ringshine(const scene *S, uint32_t index, v3 origin, v3 normal, int last_vertex, uint32_t *rng,
                    const oracle_direction *D, v3 *dshine) {
    if (dshine) *dshine = V(0, 0, 0);
    const sg_sphere *body = &S->b[index];
    if (body->ring_params[0] <= body->ring_plane[3] || body->ring_params[1] <= 0.0f) return V(0, 0, 0);
    v3 n = b_pole(S, index);
    real inner = body->ring_plane[3] * body->ring_plane[3];
    real outer = body->ring_params[0] * body->ring_params[0];
    real radius = r_sqrt(mixf(inner, outer, rnd(S, rng))) * body->radius;
    real phi = TAU_F * rnd(S, rng);
    v3 point = vmul(basis_direction(n, r_cos(phi), r_sin(phi), 0.0f), radius);
    v3 offset = vsub(point, origin);
    real distance2 = vdot(offset, offset);
    real distance = r_sqrt(distance2);
    v3 direction = vdivs(offset, distance);
    real cos_surface = vdot(normal, direction);
    real cos_ring = r_fabs(vdot(direction, n));
    if (cos_surface <= 0.0f || cos_ring < 1.0e-6f) return V(0, 0, 0);
    ray_t blocker_ray = {origin, direction, index};
    hit_t blocker = sphere_hit(S, blocker_ray, index);
    if (blocker.index != MISS && blocker.distance < distance) return V(0, 0, 0);
    optics_t optics = ring_optics(S, index, point);
    if (optics.tau == 0.0f) return V(0, 0, 0);
    optics_t doptics = ring_optics_dot(S, D, index, point);
    real mu_out = vdot(vneg(direction), n);
    v3 shine = V(0, 0, 0), dsum = V(0, 0, 0);
    uint32_t count = light_count(S);
    for (uint32_t slot = 0; slot < count; slot++) {
        uint32_t i = light_index(S, slot);
        if (b_emissive(S, i) < 0.5f) continue;
        ray_t from_ring = {point, n, index};
        light_sample light = sample_light(S, from_ring, i, rng);
        real mu_in = vdot(light.dir, n);
        ring_hit_t rh = {0.0f, index, point};
        ray_t shadow = ring_origin(S, rh, light.dir);
        real visibility = light_visibility(S, shadow, i);
        shine = vadd(shine, vmul(vmulv(ring_bsdf(optics, mu_out, mu_in), b_color(S, i)),
                                 r_fabs(mu_in) * visibility / light.pdf));
        if (D) {
            v3 bsdf = ring_bsdf(optics, mu_out, mu_in);
            v3 dbsdf = ring_bsdf_dot(optics, doptics, mu_out, mu_in);
            real dvis = light_visibility_dot(S, D, shadow, i, visibility);
            v3 dterm = vadd(vmul(vadd(vmulv(dbsdf, b_color(S, i)), vmulv(bsdf, dir_body_color(D, i))),
                                 r_fabs(mu_in) * visibility / light.pdf),
                            vmul(vmulv(bsdf, b_color(S, i)), r_fabs(mu_in) * dvis / light.pdf));
            dsum = vadd(dsum, dterm);
        }
    }
    real pdf = distance2 / (ring_area(S, index) * cos_ring);
    real weight = power_weight(pdf, cos_surface / PI_F);
    if (last_vertex) weight = 1.0f;
    if (dshine) *dshine = vmul(dsum, cos_surface * weight / (PI_F * pdf));
    return vmul(shine, cos_surface * weight / (PI_F * pdf));
}

/* point_disc_hit: pathtrace.wgsl:1308-1333 */
static hit_t point_disc_hit(const scene *S, ray_t ray, hit_t closest, real *scale, uint32_t *rng) {
    hit_t result = closest;
    real total = 0.0f;
    real pixel = 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
    real angle = clampf_(POINT_DISC_RADIUS, 0.7f * pixel, STAR_DOT_PIXELS * pixel);
    uint32_t host = (uint32_t)S->s->g.atmo_params[3] - 1u;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (i == host || S->s->g.ground_north[3] == (real)(i + 1u)) continue;
        real radius = b_radius(S, i);
        real drawn = angle * vlength(relative_center(S, ray, i));
        if (radius <= 0.0f || drawn <= radius) continue;
        hit_t hit = sphere_hit_radius(S, ray, i, drawn);
        if (hit.distance < closest.distance) {
            real ratio = (radius / drawn) * (radius / drawn);
            total += ratio;
            if (rnd(S, rng) * total < ratio) result = hit;
        }
    }
    if (total > 0.0f) *scale = total;
    return result;
}

/* point_gain: pathtrace.wgsl:1341-1345 */
static real point_gain(const scene *S, real extent, real distance) {
    real pixel = 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
    real pixels = 2.0f * extent / maxf_(distance, 1.0e-30f) / pixel;
    return mixf(S->s->background[3], 1.0f, smoothstepf(1.0f, 3.0f, pixels));
}

/* ---------------------------------------------------------------- */
/* Surface albedo (pathtrace.wgsl:338-389, :897-925)                 */
/* ---------------------------------------------------------------- */
static real hash31(v3 p) {
    v3 q = V(fractf(p.x * 0.1031f), fractf(p.y * 0.1030f), fractf(p.z * 0.0973f));
    real d = vdot(q, V(q.y + 33.33f, q.x + 33.33f, q.z + 33.33f));
    q = V(q.x + d, q.y + d, q.z + d);
    return fractf((q.x + q.y) * q.z);
}
static real vnoise(v3 p) {
    v3 i = V(r_floor(p.x), r_floor(p.y), r_floor(p.z));
    v3 f = vsub(p, i);
    v3 u = V(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y), f.z * f.z * (3.0f - 2.0f * f.z));
    real a = mixf(hash31(i), hash31(vadd(i, V(1, 0, 0))), u.x);
    real b = mixf(hash31(vadd(i, V(0, 1, 0))), hash31(vadd(i, V(1, 1, 0))), u.x);
    real c = mixf(hash31(vadd(i, V(0, 0, 1))), hash31(vadd(i, V(1, 0, 1))), u.x);
    real d = mixf(hash31(vadd(i, V(0, 1, 1))), hash31(vadd(i, V(1, 1, 1))), u.x);
    return mixf(mixf(a, b, u.y), mixf(c, d, u.y), u.z);
}
/* ---------------------------------------------------------------- */
/* Procedural surface styles 1-6 (pathtrace.wgsl:357-895)            */
/* ---------------------------------------------------------------- */
/* Transcendentals are evaluated in double and rounded to f32 (the   */
/* CUDA path does the same): the hash lattice amplifies any last-bit  */
/* difference of a noise coordinate, so both sides must agree bit for */
/* bit, and a correctly rounded value is the one both can produce.    */
static inline real sin_d(real x) { return (real)sin((double)x); }
static inline real cos_d(real x) { return (real)cos((double)x); }
static inline real atan2_d(real y, real x) { return (real)atan2((double)y, (double)x); }
static inline real exp_d(real x) { return (real)exp((double)x); }
static inline real pow_d(real x, real y) { return (real)pow((double)x, (double)y); }
static inline v3 vsplat(real s) { return V(s, s, s); }
static inline v3 vadds(v3 a, real s) { return V(a.x + s, a.y + s, a.z + s); }
static inline v3 vsubs(v3 a, real s) { return V(a.x - s, a.y - s, a.z - s); }
static inline v3 vmix(v3 a, v3 b, real t) { return V(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }
static inline v3 vfloor(v3 a) { return V(r_floor(a.x), r_floor(a.y), r_floor(a.z)); }
static inline real stepf(real edge, real x) { return x >= edge ? 1.0f : 0.0f; }

/* fbm: pathtrace.wgsl:357-373 (the octave rotation is a column matrix). */
static real fbm(v3 p, uint32_t octaves) {
    real amplitude = 0.5f, sum = 0.0f, norm = 0.0f;
    for (uint32_t octave = 0; octave < octaves; octave++) {
        sum += amplitude * vnoise(p);
        norm += amplitude;
        v3 r = V((0.0f * p.x + -1.6f * p.y) + -1.2f * p.z, (1.6f * p.x + 0.72f * p.y) + -0.96f * p.z,
                 (1.2f * p.x + -0.96f * p.y) + 1.28f * p.z);
        p = vadd(r, V(17.3f, 5.1f, 11.7f));
        amplitude *= 0.5f;
    }
    return sum / norm;
}
/* seed_offset: pathtrace.wgsl:384-389 */
static v3 seed_offset(real seed) {
    return vmul(V(hash31(V(seed, 1.0f, 7.0f)), hash31(V(3.0f, seed, 5.0f)), hash31(V(9.0f, 2.0f, seed))), 512.0f);
}
static inline v3 body_field(const sg_sphere *b, const float *f) { (void)b; return V(f[0], f[1], f[2]); }

/* gas_giant_albedo: pathtrace.wgsl:394-472 */
static v3 gas_giant_albedo(const sg_sphere *body, v3 local) {
    v3 off = seed_offset(body->axis_y[3]);
    v3 zone = body_field(body, body->color), belt = body_field(body, body->surface_color);
    real turbulence = body->surface_color[3];
    real bands = body->surface_params[0];
    uint32_t storms = (uint32_t)(body->surface_params[1] + 0.5f);
    v3 q = local;
    real masks[3] = {0, 0, 0}, rims[3] = {0, 0, 0};
    for (uint32_t k = 0; k < storms && k < 3u; k++) {
        real fk = (real)k;
        real lat = (hash31(vadd(off, V(7.1f * fk, 1.3f, 2.9f))) - 0.5f) * 1.1f;
        real lon = hash31(vadd(off, V(3.7f, 5.3f * fk, 8.1f))) * TAU_F;
        real size = (k == 0u ? 0.11f : 0.05f) * (0.8f + 0.4f * hash31(vadd(off, V(fk, 9.0f, 4.0f))));
        v3 centre = V(cos_d(lat) * cos_d(lon), cos_d(lat) * sin_d(lon), sin_d(lat));
        if (vdot(q, centre) <= 0.0f) continue;
        v3 east = V(-sin_d(lon), cos_d(lon), 0.0f);
        v3 north = vcross(centre, east);
        real dx = vdot(vsub(q, centre), east) / (2.0f * size);
        real dy = vdot(vsub(q, centre), north) / size;
        real e = r_sqrt(dx * dx + dy * dy);
        real influence = 1.0f - smoothstepf(0.0f, 2.4f, e);
        real angle = (lat < 0.0f ? 3.2f : -3.2f) * influence * influence;
        real c = cos_d(angle), s = sin_d(angle);
        real rx = c * dx - s * dy;
        real ry = s * dx + c * dy;
        q = vnormalize(vadd(vadd(q, vmul(east, (rx - dx) * 2.0f * size)), vmul(north, (ry - dy) * size)));
        real ragged = e + 0.25f * (fbm(vadd(vmul(q, 18.0f), off), 3) - 0.5f);
        masks[k] = 1.0f - smoothstepf(0.7f, 1.0f, ragged);
        rims[k] = smoothstepf(0.75f, 1.0f, ragged) * (1.0f - smoothstepf(1.0f, 1.35f, ragged));
    }
    v3 p = vadd(V(q.x * 2.2f, q.y * 2.2f, q.z * 9.0f), off);
    real warp1 = fbm(p, 5) - 0.5f;
    real warp2 = fbm(vadds(vadd(vmul(p, 2.1f), V(5.2f, 1.3f, 7.7f)), 4.0f * warp1), 5) - 0.5f;
    real lat = q.z + 0.07f * sin_d(3.0f * PI_F * q.z + off.z) + 0.04f * sin_d(5.0f * PI_F * q.z + off.y);
    real shear = 0.35f + 0.65f * r_fabs(cos_d(PI_F * bands * lat + off.x));
    real lon = atan2_d(q.y, q.x);
    real ripple = sin_d(lon * (9.0f + r_floor(bands)) + 6.0f * warp1 + off.y) * 0.5f +
                   sin_d(lon * 23.0f + 9.0f * warp2 + off.z) * 0.25f;
    real mu = lat + turbulence * shear * (0.16f * warp1 + 0.10f * warp2 + 0.025f * ripple);
    real wave = 0.5f + 0.5f * sin_d(PI_F * bands * mu + off.x);
    real irregular = fbm(V(mu * bands * 1.7f, off.y, off.z), 3);
    real profile = 0.5f * wave + 0.5f * irregular;
    real tone = fbm(V(mu * bands * 0.9f, off.z, off.x), 2);
    real fine = fbm(vadds(vadd(V(q.x * 7.0f, q.y * 7.0f, q.z * 70.0f), off), 3.0f * warp2), 4);
    real eddies = fbm(vadd(vmul(p, 5.0f), vmul(V(warp1, warp2, warp1), 6.0f)), 4);
    v3 color = vmix(belt, zone, smoothstepf(0.3f, 0.75f, profile));
    color = vmix(color, vmulv(color, vadds(vmul(color, 0.5f), 0.55f)), smoothstepf(0.35f, 0.75f, tone) * 0.8f);
    color = vmul(color, (0.78f + 0.44f * fine) * (0.9f + 0.2f * eddies));
    real polar = smoothstepf(0.55f, 0.92f, r_fabs(local.z));
    color = vmix(color, vmul(vmix(zone, belt, 0.55f), 0.8f + 0.2f * fine), polar * 0.8f);
    for (uint32_t k = 0; k < storms && k < 3u; k++) {
        v3 tint = k == 0u ? vmul(vmulv(belt, belt), 1.5f) : vmul(zone, 1.15f);
        real core = 1.0f - 0.25f * (1.0f - smoothstepf(0.0f, 0.6f, masks[k] - rims[k]));
        color = vmix(color, vmul(vmul(tint, 0.7f + 0.6f * fine), core), masks[k] * 0.92f);
        color = vmix(color, vmul(zone, 1.1f), rims[k] * 0.45f);
    }
    return color;
}

/* surface_gaussian, hash33, ridge, maria, cell_centre: pathtrace.wgsl:477-516 */
static inline real surface_gaussian(real distance) { return exp_d(-(distance * distance)); }
static v3 hash33(v3 p) {
    return V(hash31(p), hash31(vadd(p, V(19.1f, 7.3f, 3.7f))), hash31(vadd(p, V(5.9f, 31.7f, 11.3f))));
}
static inline real ridge(real n, real width) { return 1.0f - smoothstepf(0.0f, width, r_fabs(n - 0.5f)); }
static real maria(v3 q, v3 off) {
    real warp = fbm(vadd(vmul(q, 2.0f), off), 4) - 0.5f;
    return smoothstepf(0.5f, 0.56f, fbm(vadds(vadd(vmul(q, 1.2f), off), 1.5f * warp), 5));
}
static int cell_centre(v3 cell, v3 key, real scale, v3 off, v3 *centre_out) {
    for (uint32_t t = 0; t < 3u; t++) {
        v3 centre = vnormalize(vsub(vadd(cell, hash33(vadds(key, (real)t * 17.0f))), off));
        v3 f = vfloor(vadd(vmul(centre, scale), off));
        if (f.x == cell.x && f.y == cell.y && f.z == cell.z) {
            *centre_out = centre;
            return 1;
        }
    }
    return 0;
}
static inline v3 corner(v3 base, uint32_t i) {
    return vadd(base, V((real)(i & 1u), (real)((i >> 1u) & 1u), (real)((i >> 2u) & 1u)));
}

/* crater_layer: pathtrace.wgsl:527-633. state = (floor darkness, relief). */
static void crater_layer(v3 q, real scale, real density, v3 off, v3 body_off, real flood, real contrast,
                         real rays, real state[2]) {
    v3 p = vadd(vmul(q, scale), off);
    v3 base = vfloor(vsubs(p, 0.5f));
    uint32_t slots[6];
    real ages[6];
    v3 centres[6];
    uint32_t count = 0;
    for (uint32_t i = 0; i < 16u; i++) {
        v3 grid = corner(base, i);
        v3 a = vsub(grid, p), b = vsubs(vsub(p, grid), 1.0f);
        v3 gap = V(maxf_(maxf_(a.x, b.x), 0.0f), maxf_(maxf_(a.y, b.y), 0.0f), maxf_(maxf_(a.z, b.z), 0.0f));
        if (vdot(gap, gap) > 0.2343f) continue;
        v3 key = vadds(grid, (real)(i >> 3u) * 1000.0f);
        if (hash31(vadd(key, V(71.3f, 3.1f, 9.7f))) > density) continue;
        v3 found;
        if (!cell_centre(grid, key, scale, off, &found)) continue;
        real size = hash31(vadd(key, V(3.1f, 8.3f, 1.7f)));
        real radius = (0.06f + 0.16f * size * size) / scale;
        if (vlength(vsub(q, found)) > 2.2f * radius) continue;
        real age = hash31(vadd(key, V(29.0f, 61.0f, 7.0f)));
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
    real floor_shade = 1.0f, relief = state[1];
    for (uint32_t k = 0; k < count; k++) {
        uint32_t i = slots[k];
        v3 cell = vadds(corner(base, i), (real)(i >> 3u) * 1000.0f);
        v3 centre = centres[k];
        real size = hash31(vadd(cell, V(3.1f, 8.3f, 1.7f)));
        real radius = (0.06f + 0.16f * size * size) / scale;
        v3 offset = vsub(q, centre);
        real d = vlength(offset) / radius;
        v3 east = vcross(V(0.0f, 0.0f, 1.0f), centre);
        east = vdivs(east, maxf_(vlength(east), 1.0e-4f));
        v3 north = vcross(centre, east);
        real angle = atan2_d(vdot(offset, north), vdot(offset, east));
        v3 phase = vmul(hash33(vadd(cell, V(41.0f, 5.0f, 23.0f))), TAU_F);
        real wobble = 0.025f * (sin_d(3.0f * angle + phase.x) + sin_d(5.0f * angle + phase.y) +
                                 0.6f * sin_d(8.0f * angle + phase.z));
        real r = d + wobble;
        floor_shade = minf_(floor_shade, 1.0f - 0.18f * contrast * (1.0f - smoothstepf(0.55f, 0.9f, r)));
        real rim = 0.22f * contrast * surface_gaussian((r - 1.0f) / 0.13f);
        real footprint = 1.0f - smoothstepf(1.1f, 1.3f, r);
        relief = mixf(relief, rim, footprint);
        real blanket = (1.0f - smoothstepf(1.0f, 1.9f, r)) * (1.0f - footprint);
        relief = mixf(relief, 0.0f, blanket * 0.3f) + 0.1f * contrast * blanket;
        real fresh = hash31(vadd(cell, V(13.0f, 2.0f, 5.0f)));
        if (rays > 0.0f && fresh > 0.82f) {
            real streaks = pow_d(vnoise(V(cos_d(angle) * 9.0f, sin_d(angle) * 9.0f, fresh * 40.0f)), 3.0f);
            relief += contrast * (rays * 0.9f * streaks * (1.0f - smoothstepf(1.0f, 2.2f, d)) * stepf(0.9f, d) +
                                  rays * 0.25f * (1.0f - smoothstepf(0.0f, 1.0f, d)));
        }
    }
    state[0] *= floor_shade;
    state[1] = relief;
}

/* craters: pathtrace.wgsl:636-647 */
static real craters(v3 q, real density, v3 off, real flood, real contrast, real rays) {
    if (density <= 0.0f) return 1.0f;
    real state[2] = {1.0f, 0.0f};
    crater_layer(q, 1.5f, density, off, off, flood, contrast, rays, state);
    crater_layer(q, 3.5f, density, vadds(off, 101.0f), off, flood, contrast, rays * 0.8f, state);
    crater_layer(q, 8.0f, density, vadds(off, 203.0f), off, flood, contrast * 0.85f, rays * 0.5f, state);
    crater_layer(q, 18.0f, density, vadds(off, 307.0f), off, 0.0f, contrast * 0.7f, 0.0f, state);
    crater_layer(q, 40.0f, density, vadds(off, 401.0f), off, 0.0f, contrast * 0.55f, 0.0f, state);
    return state[0] * (1.0f + state[1]);
}

/* polar_caps: pathtrace.wgsl:650-656 */
static real polar_caps(v3 q, real extent, v3 off) {
    if (extent <= 0.0f) return 0.0f;
    real edge = 1.0f - extent + 0.12f * (fbm(vadd(vmul(q, 5.0f), off), 5) - 0.5f) +
                 0.05f * (fbm(vadd(vmul(q, 18.0f), off), 3) - 0.5f);
    return smoothstepf(edge - 0.015f, edge + 0.015f, r_fabs(q.z));
}

/* cratered_albedo: pathtrace.wgsl:660-669 */
static v3 cratered_albedo(const sg_sphere *body, v3 q) {
    v3 off = seed_offset(body->axis_y[3]);
    real mare = maria(q, off);
    real grain = fbm(vadd(vmul(q, 45.0f), off), 3);
    v3 color = vmix(body_field(body, body->color), body_field(body, body->surface_color), mare);
    color = vmul(color, 0.9f + 0.2f * grain);
    return vmul(color, craters(q, body->surface_color[3], off, 1.0f, 1.0f, 1.0f));
}

/* rocky_albedo: pathtrace.wgsl:673-687 */
static v3 rocky_albedo(const sg_sphere *body, v3 q) {
    v3 off = seed_offset(body->axis_y[3]);
    v3 base = vadd(vmul(q, 1.8f), off);
    v3 warp = vsubs(V(fbm(base, 4), fbm(vadds(base, 7.0f), 4), 0.0f), 0.5f);
    real dark = smoothstepf(0.5f, 0.64f, fbm(vadd(vadd(vmul(q, 2.2f), off), V(2.0f * warp.x, 2.0f * warp.y, warp.x)), 6));
    real tone = fbm(vadds(vadd(vmul(q, 5.0f), off), 3.0f), 4);
    v3 color = vmix(body_field(body, body->color), body_field(body, body->surface_color), dark * 0.85f);
    color = vmul(color, 0.85f + 0.3f * tone);
    real streak = fbm(vadds(vadd(V(q.x * 4.0f, q.y * 4.0f, q.z * 18.0f), off), 9.0f), 3);
    color = vmul(color, 0.95f + 0.1f * streak);
    color = vmul(color, craters(q, body->surface_color[3], off, 0.0f, 0.45f, 0.0f));
    real ice = polar_caps(q, body->surface_params[0], off);
    return vmix(color, V(0.92f, 0.92f, 0.94f), ice);
}

/* ice_plates: pathtrace.wgsl:691-708 */
static v3 ice_plates(v3 p) {
    v3 base = vfloor(p);
    real nearest = 10.0f, second = 10.0f, tone = 0.0f;
    for (int i = 0; i < 27; i++) {
        v3 cell = vadd(base, V((real)(i % 3 - 1), (real)((i / 3) % 3 - 1), (real)(i / 9 - 1)));
        v3 delta = vsub(vadd(vadds(cell, 0.2f), vmul(hash33(cell), 0.6f)), p);
        real d = vdot(delta, delta);
        if (d < nearest) {
            second = nearest;
            nearest = d;
            tone = hash31(vadds(cell, 57.0f));
        } else {
            second = minf_(second, d);
        }
    }
    return V(r_sqrt(nearest), r_sqrt(second) - r_sqrt(nearest), tone);
}

/* icy_albedo: pathtrace.wgsl:714-766 */
static v3 icy_albedo(const sg_sphere *body, v3 q) {
    v3 off = seed_offset(body->axis_y[3]);
    v3 ice = body_field(body, body->color);
    v3 rust = vmulv(body_field(body, body->surface_color), V(0.72f, 0.62f, 0.56f));
    v3 b = vadd(vmul(q, 3.1f), off);
    v3 warp = vsubs(V(fbm(vadds(b, 11.0f), 3), fbm(vadds(b, 23.0f), 3), fbm(vadds(b, 37.0f), 3)), 0.5f);
    real terrain = fbm(vadd(vadd(vmul(q, 4.2f), off), warp), 5);
    real rubble = fbm(vadd(vadd(vmul(q, 85.0f), off), vmul(warp, 7.0f)), 4);
    real chaos = smoothstepf(0.42f, 0.65f, terrain + 0.14f * (rubble - 0.5f));
    v3 plates = ice_plates(vadd(vadd(vmul(q, 72.0f), off), vmul(warp, 4.0f)));
    real seams = 1.0f - smoothstepf(0.015f, 0.07f, plates.y);
    real dust = chaos * (0.2f + 0.46f * rubble + 0.18f * plates.z);
    v3 color = vmix(ice, rust, dust);
    color = vmix(color, vmul(rust, 0.8f), seams * chaos * 0.35f);
    real ridged_plain = ridge(fbm(vadds(vadd(vmul(q, 34.0f), off), 83.0f), 3), 0.025f);
    color = vmix(color, rust, ridged_plain * (0.1f + 0.14f * chaos));
    color = vmul(color, 0.87f + 0.22f * fbm(vadd(vmul(q, 180.0f), off), 3));
    v3 warped = vadd(q, vmul(warp, 0.1f));
    real roughness = 0.0015f * (rubble - 0.5f);
    real shoulder = 0.0f, fissure = 0.0f, fresh_ridge = 0.0f;
    for (uint32_t i = 0; i < 64u; i++) {
        v3 h = hash33(vadd(off, V((real)i * 3.7f, 1.0f, 2.0f)));
        v3 family = hash33(vadd(off, V((real)(i / 8u) * 17.3f, 21.0f, 7.0f)));
        v3 n = vnormalize(vadd(vsubs(vmul(family, 2.0f), 1.0f), vmul(vsubs(vmul(h, 2.0f), 1.0f), 0.28f)));
        real shift = (hash31(vadd(off, V((real)i, 9.0f, 4.0f))) - 0.5f) * 1.4f;
        real width = (i < 10u ? 0.0015f + 0.0022f * h.z : 0.0005f + 0.0011f * h.z) *
                      (0.65f + 0.8f * vnoise(vadd(vmul(q, 17.0f), vmul(h, 29.0f))));
        real bend = 0.03f * (vnoise(vadd(vmul(q, 6.0f), vmul(family, 31.0f))) - 0.5f) +
                     0.008f * (vnoise(vadd(vmul(q, 24.0f), vmul(family, 37.0f))) - 0.5f);
        real dist = r_fabs(vdot(warped, n) - shift + roughness + bend);
        real along = smoothstepf(0.28f, 0.62f, vnoise(vadd(vmul(q, 3.5f), vmul(h, 50.0f))));
        shoulder = maxf_(shoulder, (1.0f - smoothstepf(width, width * 4.0f, dist)) * along);
        real double_ridge = r_fabs(dist - width * 0.85f);
        real single = 1.0f - smoothstepf(width * 0.25f, width, dist);
        real paired = 1.0f - smoothstepf(width * 0.15f, width * 0.55f, double_ridge);
        fissure = maxf_(fissure, (i < 10u ? paired : single) * along);
        fresh_ridge = maxf_(fresh_ridge,
                            (1.0f - smoothstepf(width * 0.15f, width * 0.35f, r_fabs(dist - width * 1.8f))) * along);
    }
    color = vmix(color, rust, shoulder * 0.17f);
    color = vmix(color, vmul(rust, 0.7f), fissure * 0.8f);
    color = vmix(color, ice, fresh_ridge * 0.13f);
    return vmul(color, craters(q, body->surface_color[3] * 0.2f, off, 0.0f, 0.3f, 0.4f));
}

/* volcanic_albedo: pathtrace.wgsl:770-850 */
static v3 volcanic_albedo(const sg_sphere *body, v3 q) {
    v3 off = seed_offset(body->axis_y[3]);
    v3 sulphur = body_field(body, body->color), deposit = body_field(body, body->surface_color);
    v3 b = vadd(vmul(q, 4.7f), off);
    v3 warp = vsubs(V(fbm(b, 3), fbm(vadds(b, 19.0f), 3), fbm(vadds(b, 41.0f), 3)), 0.5f);
    real terrain = fbm(vadd(vadd(vmul(q, 10.0f), off), vmul(warp, 2.0f)), 6);
    real weathered = smoothstepf(0.38f, 0.65f, fbm(vadds(vadd(vmul(q, 3.7f), off), 11.0f), 5));
    real fine = fbm(vadd(vadd(vmul(q, 90.0f), off), vmul(warp, 3.0f)), 4);
    v3 crust = vmix(vmulv(sulphur, V(0.43f, 0.51f, 0.6f)), deposit, 0.12f);
    v3 color = vmul(sulphur, 0.7f + 0.5f * terrain);
    color = vmix(color, crust, weathered * (0.45f + 0.5f * terrain));
    real frost = smoothstepf(0.38f, 0.74f, fbm(vadd(vadds(vadd(vmul(q, 6.0f), off), 29.0f), warp), 5) + 0.2f * (fine - 0.5f));
    v3 frost_color = vmix(sulphur, V(0.72f, 0.7f, 0.62f), 0.8f);
    color = vmix(color, frost_color, frost * 0.7f);
    real flow_edges = ridge(fbm(vadd(vadd(vmul(q, 35.0f), off), vmul(warp, 2.0f)), 4), 0.025f);
    color = vmix(color, crust, flow_edges * weathered * 0.4f);
    color = vmul(color, (0.82f + 0.32f * fine) * (0.94f + 0.13f * fbm(vadd(vmul(q, 210.0f), off), 3)));
    real dark = 0.0f, ash = 0.0f, red = 0.0f, white = 0.0f;
    real density = body->surface_color[3];
    real scale = 5.5f;
    v3 p = vadds(vadd(vmul(q, scale), off), 300.0f);
    v3 base = vfloor(p);
    for (int i = 0; i < 27; i++) {
        v3 cell = vadd(base, V((real)(i % 3 - 1), (real)((i / 3) % 3 - 1), (real)(i / 9 - 1)));
        if (hash31(vadd(cell, V(4.0f, 41.0f, 9.0f))) > 0.6f * density) continue;
        v3 centre;
        if (!cell_centre(cell, cell, scale, vadds(off, 300.0f), &centre)) continue;
        real size = hash31(vadd(cell, V(8.0f, 1.0f, 3.0f)));
        real radius = (0.025f + 0.11f * size * size * size) / scale;
        v3 offset = vsub(q, centre);
        real reach = vlength(offset) * scale;
        if (reach > 0.95f) continue;
        real cutoff = 1.0f - smoothstepf(0.75f, 0.95f, reach);
        v3 tangent = vcross(centre, V(0.37f, 0.83f, 0.41f));
        v3 east = vdivs(tangent, maxf_(vlength(tangent), 1.0e-5f));
        v3 north = vcross(centre, east);
        real angle = TAU_F * hash31(vadds(cell, 91.0f));
        real ux = vdot(offset, east) / radius, uy = vdot(offset, north) / radius;
        real ca = cos_d(angle), sa = sin_d(angle);
        real uvx = ux * ca - uy * sa, uvy = ux * sa + uy * ca;
        real ragged = fbm(vadd(V(uvx * 2.7f, uvy * 2.7f, 0.0f), vmul(cell, 7.0f)), 3) - 0.5f;
        real sx = uvx * (1.0f / (0.65f + 0.9f * size)), sy = uvy * 1.0f;
        real d = r_sqrt(sx * sx + sy * sy) + 0.42f * ragged;
        real pit = 1.0f - smoothstepf(0.68f, 0.86f, d);
        real age = hash31(vadds(cell, 31.0f));
        real fx = uvx - (0.2f + 2.3f * age), fy = uvy - 0.35f * sin_d(uvx * 1.3f + angle);
        real gx = fx * (0.75f - 0.48f * age), gy = fy * (0.85f + 0.35f * size);
        real flow_shape = r_sqrt(gx * gx + gy * gy) + 0.65f * ragged +
                           0.35f * (fbm(vadd(V(uvx * 1.8f, uvy * 1.8f, 0.0f), vmul(cell, 3.0f)), 4) - 0.5f);
        real flow = (1.0f - smoothstepf(0.72f, 0.9f, flow_shape)) * smoothstepf(0.35f, 0.85f, age) * 0.85f;
        dark = maxf_(dark, maxf_(pit, flow) * cutoff);
        real plume = hash31(vadd(cell, V(2.0f, 6.0f, 17.0f)));
        real hx = (uvx - 0.5f) * 0.16f, hy = (uvy - 0.3f) * 0.23f;
        real halo = exp_d(-(hx * hx + hy * hy)) * cutoff;
        ash = maxf_(ash, halo * (0.25f + 0.35f * age));
        white = maxf_(white, halo * stepf(0.45f, plume) * (1.0f - stepf(0.83f, plume)));
        real apron = surface_gaussian((r_sqrt(uvx * uvx + uvy * uvy) + ragged - 3.5f) / 1.6f) *
                      (0.25f + 0.75f * smoothstepf(-1.5f, 2.0f, uvy));
        red = maxf_(red, apron * stepf(0.83f, plume) * cutoff);
    }
    color = vmix(color, vmul(crust, 0.7f), ash * 0.45f);
    color = vmix(color, frost_color, white * 0.4f);
    color = vmix(color, vmulv(deposit, V(0.85f, 0.7f, 0.65f)), red * 0.6f);
    return vmix(color, V(0.035f, 0.032f, 0.026f), dark * 0.96f);
}

/* terran_albedo: pathtrace.wgsl:854-895 */
static v3 terran_albedo(const sg_sphere *body, v3 q) {
    v3 off = seed_offset(body->axis_y[3]);
    v3 land_base = body_field(body, body->color), ocean = body_field(body, body->surface_color);
    v3 b = vadd(vmul(q, 1.5f), off);
    v3 warp = vsubs(V(fbm(b, 4), fbm(vadds(b, 13.0f), 4), fbm(vadds(b, 29.0f), 4)), 0.5f);
    real height = fbm(vadd(vadd(vmul(q, 1.1f), off), vmul(warp, 0.9f)), 7);
    real sea = 0.5f + (body->surface_params[1] - 0.5f) * 0.3f;
    real coast = smoothstepf(sea, sea + 0.004f, height);
    real shallow = 1.0f - smoothstepf(sea - 0.04f, sea, height);
    v3 water = vmix(vadd(vmul(ocean, 1.8f), V(0.0f, 0.04f, 0.05f)), ocean, shallow);
    real moisture = fbm(vadds(vadd(vmul(q, 3.0f), off), 41.0f), 5) + 0.25f * (r_fabs(q.z) - 0.35f);
    v3 green = vmulv(land_base, V(0.45f, 0.62f, 0.38f));
    v3 land = vmix(land_base, green, smoothstepf(0.45f, 0.6f, moisture));
    real altitude = smoothstepf(sea + 0.08f, sea + 0.2f, height);
    land = vmix(land, V(0.42f, 0.38f, 0.34f), altitude * 0.6f);
    land = vmix(land, V(0.9f, 0.9f, 0.92f), smoothstepf(sea + 0.19f, sea + 0.24f, height));
    land = vmul(land, 0.88f + 0.24f * fbm(vadd(vmul(q, 25.0f), off), 3));
    v3 color = vmix(water, land, coast);
    real ice = polar_caps(q, body->surface_params[0], off);
    color = vmix(color, V(0.9f, 0.92f, 0.95f), ice);
    real cover = body->surface_params[2];
    if (cover > 0.0f) {
        v3 c1 = vadd(vmul(q, 1.6f), off);
        v3 w1 = vsubs(V(fbm(vadds(c1, 77.0f), 4), fbm(vadds(c1, 91.0f), 4), 0.5f), 0.5f);
        v3 c2 = vadd(vadd(vmul(q, 4.0f), off), vmul(w1, 3.0f));
        v3 w2 = vsubs(V(fbm(c2, 4), fbm(vadd(vadds(vadd(vmul(q, 4.0f), off), 17.0f), vmul(w1, 3.0f)), 4), 0.5f), 0.5f);
        v3 cq = vadd(vadd(vadd(V(q.x * 2.5f, q.y * 2.5f, q.z * 7.0f), off), vmul(w1, 2.5f)), vmul(w2, 1.2f));
        real cloud = fbm(cq, 7);
        real lat = r_fabs(q.z);
        real belts = 0.06f * (surface_gaussian(lat / 0.12f) + surface_gaussian((lat - 0.72f) / 0.15f)) -
                      0.04f * surface_gaussian((lat - 0.42f) / 0.1f);
        real threshold = 0.62f - 0.22f * cover - belts;
        real mask = smoothstepf(threshold - 0.04f, threshold + 0.14f, cloud);
        color = vmix(color, V(0.93f, 0.94f, 0.96f), mask * 0.95f);
    }
    return color;
}

/* surface_albedo, styles 1-6 (pathtrace.wgsl:897-910): clamped to [0, 1]. */
static v3 style_albedo(const sg_sphere *body, uint32_t style, v3 local) {
    v3 c;
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

static v3 surface_albedo_m(const scene *S, uint32_t index, v3 normal, real *mottle_out) {
    const sg_sphere *body = &S->b[index];
    v3 x = V(body->axis_x[0], body->axis_x[1], body->axis_x[2]);
    v3 y = V(body->axis_y[0], body->axis_y[1], body->axis_y[2]);
    v3 local = V(vdot(normal, x), vdot(normal, y), vdot(normal, vcross(x, y)));
    uint32_t style = body->axis_x[3] >= 0.5f ? (uint32_t)(body->axis_x[3] + 0.5f) : 0u;
    if (style > 0u) {
        if (mottle_out) *mottle_out = 1.0f;
        return style_albedo(body, style, local);
    }
    real mottle = 1.0f;
    if (body->center_low[3] > 0.0f) {
        real seed = body->axis_y[3];
        v3 off = vmul(V(hash31(V(seed, 1.0f, 7.0f)), hash31(V(3.0f, seed, 5.0f)), hash31(V(9.0f, 2.0f, seed))), 512.0f);
        v3 p = vadd(vmul(local, 2.4f), off);
        real amplitude = 0.5f, noise = 0.0f;
        for (int octave = 0; octave < 5; octave++) {
            noise += amplitude * vnoise(p);
            p = vmul(p, 2.07f);
            amplitude *= 0.5f;
        }
        mottle = mixf(1.0f, 0.68f + 0.64f * noise, body->center_low[3]);
    }
    if (mottle_out) *mottle_out = mottle;
    v3 c = vmul(b_color(S, index), mottle);
    return V(clampf_(c.x, 0, 1), clampf_(c.y, 0, 1), clampf_(c.z, 0, 1));
}

static v3 surface_albedo(const scene *S, uint32_t index, v3 normal) {
    return surface_albedo_m(S, index, normal, NULL);
}

/* Tangent of surface_albedo: the colour scaled by the mottle where the
 * clamp to [0, 1] is inactive. */
static v3 surface_albedo_dot(const scene *S, const oracle_direction *D, uint32_t index, v3 normal) {
    real m = 1.0f;
    (void)surface_albedo_m(S, index, normal, &m);
    v3 c = vmul(b_color(S, index), m);
    v3 d = vmul(dir_body_color(D, index), m);
    return V(c.x > 0.0f && c.x < 1.0f ? d.x : 0.0f, c.y > 0.0f && c.y < 1.0f ? d.y : 0.0f,
             c.z > 0.0f && c.z < 1.0f ? d.z : 0.0f);
}

/* ---------------------------------------------------------------- */
/* Local landscape: ground.wgsl:14-242, :597-666; terrain.wgsl       */
/* ---------------------------------------------------------------- */
#define METRES_PER_AU 149597870700.0f
#define TERRAIN_ID SG_TERRAIN_ID

static inline v3 g_east(const scene *S) { return V(S->s->g.ground_east[0], S->s->g.ground_east[1], S->s->g.ground_east[2]); }
static inline v3 g_up(const scene *S) { return V(S->s->g.ground_up[0], S->s->g.ground_up[1], S->s->g.ground_up[2]); }
static inline v3 g_north(const scene *S) { return V(S->s->g.ground_north[0], S->s->g.ground_north[1], S->s->g.ground_north[2]); }

/* camera_origin, to_ground, from_ground, ground_origin: ground.wgsl:17-32 */
static v3 camera_origin(const scene *S, ray_t ray) {
    if (ray.anchor == MISS) return ray.offset;
    return vadd(b_center(S, ray.anchor), vadd(b_low(S, ray.anchor), ray.offset));
}
static v3 to_ground(const scene *S, v3 v) { return V(vdot(v, g_east(S)), vdot(v, g_up(S)), vdot(v, g_north(S))); }
static v3 from_ground(const scene *S, v3 v) {
    return vadd(vadd(vmul(g_east(S), v.x), vmul(g_up(S), v.y)), vmul(g_north(S), v.z));
}
static v3 ground_origin(const scene *S, ray_t ray) {
    v3 g = to_ground(S, vmul(camera_origin(S, ray), METRES_PER_AU));
    return vadd(g, V(0.0f, S->s->g.ground_east[3], 0.0f));
}
/* Rotation sines and cosines are evaluated in double and rounded to f32,
 * a rounding the CUDA path reproduces exactly (it precomputes the same
 * values per primitive on the host). */
static inline real sin_r(real angle) { return (real)sin((double)angle); }
static inline real cos_r(real angle) { return (real)cos((double)angle); }
static v3 rotate_north(v3 p, real angle) {
    real c = cos_r(angle), s = sin_r(angle);
    return V(c * p.x - s * p.y, s * p.x + c * p.y, p.z);
}
static v3 rotate_east(v3 p, real angle) {
    real c = cos_r(angle), s = sin_r(angle);
    return V(p.x, c * p.y - s * p.z, s * p.y + c * p.z);
}
static v3 rotate_up(v3 p, real angle) {
    real c = cos_r(angle), s = sin_r(angle);
    return V(c * p.x + s * p.z, p.y, -s * p.x + c * p.z);
}
/* rock_angles, rock_to_local, rock_from_local: ground.wgsl:41-61 */
static v3 rock_angles(real packed) {
    uint32_t bits = (uint32_t)packed;
    return vmul(V((real)(bits & 255u), (real)((bits >> 8) & 255u), (real)((bits >> 16) & 255u)), TAU_F / 256.0f);
}
static v3 rock_to_local(v3 p, v3 a) { return rotate_east(rotate_up(rotate_north(p, -a.z), -a.y), -a.x); }
static v3 rock_from_local(v3 p, v3 a) { return rotate_north(rotate_up(rotate_east(p, a.x), a.y), a.z); }

static inline real vcomp(v3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

/* box_interval: ground.wgsl:64-78 */
static void box_interval(v3 p, v3 d, v3 extent, real *near_, real *far_) {
    real n = -1.0e30f, f = 1.0e30f;
    for (int axis = 0; axis < 3; axis++) {
        real pa = vcomp(p, axis), da = vcomp(d, axis), ea = vcomp(extent, axis);
        if (r_fabs(da) < 1.0e-12f) {
            if (r_fabs(pa) > ea) { *near_ = 1.0e30f; *far_ = -1.0e30f; return; }
        } else {
            real a = (-ea - pa) / da;
            real b = (ea - pa) / da;
            n = maxf_(n, minf_(a, b));
            f = minf_(f, maxf_(a, b));
        }
    }
    *near_ = n;
    *far_ = f;
}

/* rock_hit: ground.wgsl:82-121, returns the distance, normal in *n */
static real rock_hit(v3 p, v3 d, v3 e, v3 *normal) {
    v3 origin = V(p.x / e.x, p.y / e.y, p.z / e.z);
    v3 direction = V(d.x / e.x, d.y / e.y, d.z / e.z);
    real near_ = -1.0e30f, far_ = 1.0e30f;
    v3 near_normal = V(0, 0, 0), far_normal = V(0, 0, 0);
    for (uint32_t face = 0; face < 14u; face++) {
        v3 n = V(0, 0, 0);
        real limit = 1.0f;
        if (face < 6u) {
            real s = (face & 1u) == 1u ? 1.0f : -1.0f;
            if (face / 2u == 0) n.x = s; else if (face / 2u == 1) n.y = s; else n.z = s;
        } else {
            uint32_t bits = face - 6u;
            n = V((bits & 1u) ? 1.0f : -1.0f, (bits & 2u) ? 1.0f : -1.0f, (bits & 4u) ? 1.0f : -1.0f);
            limit = 1.65f + 0.08f * (real)(bits % 3u);
        }
        real denominator = vdot(n, direction);
        real gap = limit - vdot(n, origin);
        if (r_fabs(denominator) < 1.0e-12f) {
            if (gap < 0.0f) return 1.0e30f;
        } else {
            real distance = gap / denominator;
            if (denominator < 0.0f && distance > near_) { near_ = distance; near_normal = V(n.x / e.x, n.y / e.y, n.z / e.z); }
            if (denominator > 0.0f && distance < far_) { far_ = distance; far_normal = V(n.x / e.x, n.y / e.y, n.z / e.z); }
        }
        if (near_ > far_) return 1.0e30f;
    }
    if (far_ <= 0.001f) return 1.0e30f;
    if (near_ > 0.001f) { *normal = vnormalize(near_normal); return near_; }
    *normal = vnormalize(far_normal);
    return far_;
}

/* Terrain layout helpers: terrain.wgsl:6-36 */
static uint32_t t_cells(const scene *S) {
    uint32_t log2 = S->s->g.ground_counts[2] >> 8;
    return log2 != 0u ? (1u << log2) : 512u;
}
static inline uint32_t t_width(uint32_t cells) { return cells + 1u; }
static inline uint32_t t_vertices(uint32_t cells) { return t_width(cells) * t_width(cells); }
static inline int t_compact(uint32_t cells) { return cells > 1024u; }
static inline uint32_t t_vertex_stride(uint32_t cells) { return t_compact(cells) ? 2u : 6u; }
static inline uint32_t t_nodes(uint32_t cells) { uint32_t leaves = cells / 2u; return (4u * leaves * leaves - 1u) / 3u; }
static inline uint32_t t_bounds(uint32_t cells) { return (t_compact(cells) ? 1u : 3u) * t_vertices(cells); }
static inline uint32_t t_cache(uint32_t cells) { return t_bounds(cells) + 2u * t_nodes(cells); }
static inline uint32_t t_vertex_cache(uint32_t cells) { return t_cache(cells) + 6u * t_nodes(cells); }
static inline uint32_t ground_theme(const scene *S) { return S->s->g.ground_counts[2] & 255u; }

size_t oracle_terrain_floats(uint32_t cells) {
    return (size_t)t_vertex_cache(cells) + (size_t)t_vertices(cells) * t_vertex_stride(cells);
}

static inline real t_scale_r(real r) { return clampf_(r / 200000.0f, 0.0001f, 1.0f); }
static inline real t_coordinate(uint32_t i, uint32_t cells, real scale) {
    real u = 2.0f * (real)i / (real)cells - 1.0f;
    return u * r_fabs(u) * 16000.0f * scale;
}
static inline real t_curvature(real px, real pz, real r) {
    real d2 = px * px + pz * pz;
    return -d2 / (r + r_sqrt(maxf_(r * r - d2, 0.0f)));
}
/* De-interleave one Morton axis (terrain.wgsl:134-140). */
static inline uint32_t compact_bits(uint32_t value) {
    uint32_t x = value & 0x55555555u;
    x = (x | (x >> 1)) & 0x33333333u;
    x = (x | (x >> 2)) & 0x0f0f0f0fu;
    x = (x | (x >> 4)) & 0x00ff00ffu;
    return (x | (x >> 8)) & 0x0000ffffu;
}
static inline uint32_t first_leading_bit(uint32_t v) { uint32_t n = 0; while (v >>= 1) n++; return n; }
static void node_of(uint32_t index, uint32_t cells, uint32_t node[4]) {
    uint32_t level = first_leading_bit(3u * index + 1u) / 2u;
    uint32_t size = cells >> level;
    uint32_t morton = index - ((1u << (2u * level)) - 1u) / 3u;
    node[0] = index;
    node[1] = compact_bits(morton) * size;
    node[2] = compact_bits(morton >> 1) * size;
    node[3] = size;
}

/* cache_terrain_geometry: terrain.wgsl:242-285 with the uncached helpers
 * :37-61 and :85-95. */
int oracle_cache_terrain(float *T, uint32_t cells, float r) {
    if (!T || cells < 2u || (cells & (cells - 1u)) != 0u) return SG_ERR_INVALID;
    real scale = t_scale_r(r);
    uint32_t width = t_width(cells), nodes = t_nodes(cells), vertices = t_vertices(cells);
    for (uint32_t index = 0; index < nodes; index++) {
        uint32_t node[4];
        node_of(index, cells, node);
        real lo_x = t_coordinate(node[1], cells, scale), lo_z = t_coordinate(node[2], cells, scale);
        real hi_x = t_coordinate(node[1] + node[3], cells, scale), hi_z = t_coordinate(node[2] + node[3], cells, scale);
        real near_x = clampf_(0.0f, lo_x, hi_x), near_z = clampf_(0.0f, lo_z, hi_z);
        real far_x = maxf_(r_fabs(lo_x), r_fabs(hi_x)), far_z = maxf_(r_fabs(lo_z), r_fabs(hi_z));
        real lower = T[t_bounds(cells) + index * 2u] * scale + t_curvature(far_x, far_z, r) - 0.02f;
        real upper = T[t_bounds(cells) + index * 2u + 1u] * scale + t_curvature(near_x, near_z, r) + 0.02f;
        float *c = T + t_cache(cells) + (size_t)index * 6u;
        c[0] = lo_x; c[1] = lower; c[2] = lo_z; c[3] = hi_x; c[4] = upper; c[5] = hi_z;
    }
    for (uint32_t index = 0; index < vertices; index++) {
        uint32_t x = index % width, z = index / width;
        real px = t_coordinate(x, cells, scale), pz = t_coordinate(z, cells, scale);
        v3 vertex = V(px, T[z * width + x] * scale + t_curvature(px, pz, r), pz);
        real denom = r_sqrt(maxf_(r * r - (px * px + pz * pz), 1.0f));
        real gx = px / denom, gz = pz / denom;
        v3 normal;
        if (t_compact(cells)) {
            uint32_t lox = x > 0 ? x - 1u : 0u, loz = z > 0 ? z - 1u : 0u;
            uint32_t hix = x + 1u < cells ? x + 1u : cells, hiz = z + 1u < cells ? z + 1u : cells;
            real dx = (T[z * width + hix] - T[z * width + lox]) /
                       ((t_coordinate(hix, cells, scale) - t_coordinate(lox, cells, scale)) / scale);
            real dz = (T[hiz * width + x] - T[loz * width + x]) /
                       ((t_coordinate(hiz, cells, scale) - t_coordinate(loz, cells, scale)) / scale);
            normal = vnormalize(V(-dx + gx, 1.0f, -dz + gz));
        } else {
            normal = vnormalize(V(-T[vertices + index] + gx, 1.0f, -T[2u * vertices + index] + gz));
        }
        float *v = T + t_vertex_cache(cells) + (size_t)index * t_vertex_stride(cells);
        if (t_compact(cells)) {
            v[0] = vertex.y;
            /* WGSL round() rounds half to even, as r_rint does. */
            real ux = r_rint(clampf_(normal.x * 0.5f + 0.5f, 0.0f, 1.0f) * 4095.0f);
            real uz = r_rint(clampf_(normal.z * 0.5f + 0.5f, 0.0f, 1.0f) * 4095.0f);
            v[1] = (real)((uint32_t)ux | ((uint32_t)uz << 12));
        } else {
            v[0] = vertex.x; v[1] = vertex.y; v[2] = vertex.z;
            v[3] = normal.x; v[4] = normal.y; v[5] = normal.z;
        }
    }
    return SG_OK;
}

/* terrain_vertex / terrain_normal: terrain.wgsl:97-115 */
static v3 t_vertex(const float *T, uint32_t cells, real scale, uint32_t x, uint32_t z) {
    const float *v = T + t_vertex_cache(cells) + (size_t)(z * t_width(cells) + x) * t_vertex_stride(cells);
    if (t_compact(cells)) return V(t_coordinate(x, cells, scale), v[0], t_coordinate(z, cells, scale));
    return V(v[0], v[1], v[2]);
}
static v3 t_normal(const float *T, uint32_t cells, uint32_t x, uint32_t z) {
    const float *v = T + t_vertex_cache(cells) + (size_t)(z * t_width(cells) + x) * t_vertex_stride(cells);
    if (t_compact(cells)) {
        uint32_t packed = (uint32_t)v[1];
        real xx = (real)(packed & 4095u) / 4095.0f * 2.0f - 1.0f;
        real zz = (real)(packed >> 12) / 4095.0f * 2.0f - 1.0f;
        return vnormalize(V(xx, r_sqrt(maxf_(1.0f - (xx * xx + zz * zz), 1.0e-6f)), zz));
    }
    return V(v[3], v[4], v[5]);
}

/* terrain_triangle: terrain.wgsl:65-81 -> (u, v, distance) */
static v3 t_triangle(v3 o, v3 d, v3 a, v3 b, v3 c) {
    v3 ab = vsub(b, a), ac = vsub(c, a);
    v3 p = vcross(d, ac);
    real determinant = vdot(ab, p);
    if (r_fabs(determinant) < 1.0e-12f) return V(0, 0, 1.0e30f);
    real inverse = 1.0f / determinant;
    v3 relative = vsub(o, a);
    real u = vdot(relative, p) * inverse;
    v3 q = vcross(relative, ab);
    real v = vdot(d, q) * inverse;
    real distance = vdot(ac, q) * inverse;
    if (u < -1.0e-6f || v < -1.0e-6f || u + v > 1.000001f || distance <= 0.001f) return V(0, 0, 1.0e30f);
    return V(u, v, distance);
}

/* terrain_interval: terrain.wgsl:118-130 */
static void t_interval(const float *T, uint32_t cells, v3 o, v3 inv, uint32_t index, real *entry, real *exit_) {
    const float *c = T + t_cache(cells) + (size_t)index * 6u;
    real lo[3] = {c[0], c[1], c[2]}, hi[3] = {c[3], c[4], c[5]};
    real oo[3] = {o.x, o.y, o.z}, ii[3] = {inv.x, inv.y, inv.z};
    real e0[3], e1[3];
    for (int k = 0; k < 3; k++) {
        int parallel = r_fabs(ii[k]) >= 1.0e29f;
        if (parallel && (oo[k] < lo[k] || oo[k] > hi[k])) { *entry = 1.0e30f; *exit_ = -1.0e30f; return; }
    }
    for (int k = 0; k < 3; k++) {
        int parallel = r_fabs(ii[k]) >= 1.0e29f;
        real a = (lo[k] - oo[k]) * ii[k];
        real b = (hi[k] - oo[k]) * ii[k];
        e0[k] = parallel ? -1.0e30f : minf_(a, b);
        e1[k] = parallel ? 1.0e30f : maxf_(a, b);
    }
    *entry = maxf_(e0[0], maxf_(e0[1], e0[2]));
    *exit_ = minf_(e1[0], minf_(e1[1], e1[2]));
}

static int is_terrain_alpine(const scene *S) { return ground_theme(S) == 3u; }

/* terrain_shading: terrain.wgsl:142-150 (alpine: steep triangles shade with
 * their flat face). */
static v3 terrain_shading(const scene *S, v3 smooth_normal, v3 a, v3 b, v3 c) {
    if (!is_terrain_alpine(S)) return smooth_normal;
    v3 face = vnormalize(vcross(vsub(b, a), vsub(c, a)));
    if (face.y < 0.0f) face = vneg(face);
    return vnormalize(vmix(smooth_normal, face, smoothstepf(0.25f, 0.5f, 1.0f - face.y)));
}

/* terrain_query: terrain.wgsl:152-234 (stack widened to 40 slots so 4096
 * cells, eleven internal levels, fit: 3 * 11 + 1 = 34 entries). */
static real t_query(const scene *S, const float *T, uint32_t cells, v3 o, v3 d, real initial_limit, int occlusion,
                     v3 *normal) {
    real limit = initial_limit;
    real result = 1.0e30f;
    real scale = t_scale_r(S->s->g.ground_up[3]);
    v3 inv = V((d.x >= 0.0f ? 1.0f : -1.0f) / maxf_(r_fabs(d.x), 1.0e-30f),
               (d.y >= 0.0f ? 1.0f : -1.0f) / maxf_(r_fabs(d.y), 1.0e-30f),
               (d.z >= 0.0f ? 1.0f : -1.0f) / maxf_(r_fabs(d.z), 1.0e-30f));
    real re, rx;
    t_interval(T, cells, o, inv, 0u, &re, &rx);
    if (re > rx || rx <= 0.001f || re >= limit) return result;
    uint32_t stack_node[40];
    real stack_t[40];
    stack_node[0] = 0u;
    stack_t[0] = maxf_(re, 0.0f);
    uint32_t count = 1;
    while (count > 0u) {
        count--;
        if (stack_t[count] >= limit) continue;
        uint32_t node[4];
        node_of(stack_node[count], cells, node);
        if (node[3] == 2u) {
            for (uint32_t z = node[2]; z < node[2] + 2u; z++) {
                for (uint32_t x = node[1]; x < node[1] + 2u; x++) {
                    EV(terrain_triangles);
                    EV(terrain_triangles);
                    v3 a = t_vertex(T, cells, scale, x, z);
                    v3 b = t_vertex(T, cells, scale, x + 1u, z);
                    v3 c = t_vertex(T, cells, scale, x, z + 1u);
                    v3 e = t_vertex(T, cells, scale, x + 1u, z + 1u);
                    v3 first = t_triangle(o, d, a, c, b);
                    v3 second = t_triangle(o, d, e, b, c);
                    if (first.z < limit) {
                        if (occlusion) { *normal = V(0, 0, 0); return first.z; }
                        v3 n = vnormalize(vadd(vadd(vmul(t_normal(T, cells, x, z), 1.0f - first.x - first.y),
                                                    vmul(t_normal(T, cells, x, z + 1u), first.x)),
                                               vmul(t_normal(T, cells, x + 1u, z), first.y)));
                        *normal = terrain_shading(S, n, a, c, b);
                        result = first.z;
                        limit = first.z;
                    }
                    if (second.z < limit) {
                        if (occlusion) { *normal = V(0, 0, 0); return second.z; }
                        v3 n = vnormalize(vadd(vadd(vmul(t_normal(T, cells, x + 1u, z + 1u), 1.0f - second.x - second.y),
                                                    vmul(t_normal(T, cells, x + 1u, z), second.x)),
                                               vmul(t_normal(T, cells, x, z + 1u), second.y)));
                        *normal = terrain_shading(S, n, e, b, c);
                        result = second.z;
                        limit = second.z;
                    }
                }
            }
        } else {
            EV(terrain_nodes);
            uint32_t children[4];
            real distances[4];
            uint32_t half_size = node[3] / 2u;
            for (uint32_t child = 0; child < 4u; child++) {
                children[child] = node[0] * 4u + child + 1u;
                real be, bx;
                t_interval(T, cells, o, inv, children[child], &be, &bx);
                distances[child] = (be <= bx && bx > 0.001f && be < limit) ? maxf_(be, 0.0f) : 1.0e30f;
                (void)half_size;
            }
            for (uint32_t i = 1; i < 4u; i++) {
                uint32_t j = i;
                while (!(j == 0u || distances[j - 1u] >= distances[j])) {
                    real dd = distances[j - 1u];
                    uint32_t cc = children[j - 1u];
                    distances[j - 1u] = distances[j];
                    children[j - 1u] = children[j];
                    distances[j] = dd;
                    children[j] = cc;
                    j--;
                }
            }
            for (uint32_t i = 0; i < 4u; i++) {
                if (distances[i] < limit && count < 40u) {
                    stack_node[count] = children[i];
                    stack_t[count] = distances[i];
                    count++;
                }
            }
        }
    }
    return result;
}

int oracle_terrain_query(const sg_settings *settings, const oracle_tables *tables, const float o[3], const float d[3],
                         float limit, int occlusion, float out[4]) {
    if (!settings || !tables || !tables->terrain) return SG_ERR_INVALID;
    scene S = {settings, NULL, tables, NULL, NULL, NULL};
    v3 n = V(0, 0, 0);
    real t = t_query(&S, tables->terrain, t_cells(&S), V(o[0], o[1], o[2]), V(d[0], d[1], d[2]), limit, occlusion, &n);
    out[0] = n.x; out[1] = n.y; out[2] = n.z; out[3] = t;
    return SG_OK;
}

/* landscape_top: ground.wgsl:244-251 */
static real landscape_top(const scene *S) {
    float top_bits;
    uint32_t bits = S->s->g.ground_counts[3];
    memcpy(&top_bits, &bits, sizeof(top_bits));
    real top = top_bits;
    if (S->s->g.ground_counts[1] != 0u && S->t && S->t->terrain)
        top = maxf_(top, S->t->terrain[t_cache(t_cells(S)) + 4u]);
    return top;
}

/* ---------------------------------------------------------------- */
/* Vegetation primitives (kinds 3 conifer, 4 grass, 5 trunk):        */
/* forest.wgsl:56-136, in the primitive's frame. (normal, distance), */
/* distance 1e30 on a miss. Strict f32, correctly rounded            */
/* transcendentals.                                                  */
/* ---------------------------------------------------------------- */
typedef struct { v3 n; real t; } veg_hit;
static veg_hit trunk_hit(v3 p, v3 d, v3 e) {
    v3 o = V(p.x / e.x, p.y / e.y, p.z / e.z);
    v3 v = V(d.x / e.x, d.y / e.y, d.z / e.z);
    veg_hit result = {V(0.0f, 0.0f, 0.0f), 1.0e30f};
    real a = v.x * v.x + v.z * v.z;
    real b = o.x * v.x + o.z * v.z;
    real c = o.x * o.x + o.z * o.z - 1.0f;
    real disc = b * b - a * c;
    if (a > 1.0e-15f && disc >= 0.0f) {
        for (uint32_t side = 0; side < 2u; side++) {
            real t = (-b + (side == 1u ? r_sqrt(disc) : -r_sqrt(disc))) / a;
            v3 q = vadd(o, vmul(v, t));
            if (t > 0.001f && t < result.t && r_fabs(q.y) <= 1.0f) {
                result.n = vnormalize(V(q.x / e.x, 0.0f / e.y, q.z / e.z));
                result.t = t;
            }
        }
    }
    if (r_fabs(v.y) > 1.0e-15f) {
        for (uint32_t side = 0; side < 2u; side++) {
            real sign_y = side == 1u ? 1.0f : -1.0f;
            real t = (sign_y - o.y) / v.y;
            v3 q = vadd(o, vmul(v, t));
            if (t > 0.001f && t < result.t && q.x * q.x + q.z * q.z <= 1.0f) {
                result.n = V(0.0f, sign_y, 0.0f);
                result.t = t;
            }
        }
    }
    return result;
}
static veg_hit conifer_hit(v3 p, v3 d, v3 e) {
    veg_hit result = trunk_hit(vadd(p, V(0.0f, e.y * 0.08f, 0.0f)), d, V(e.x * 0.065f, e.y * 0.92f, e.z * 0.065f));
    v3 o = V(p.x / e.x, p.y / e.y, p.z / e.z);
    v3 v = V(d.x / e.x, d.y / e.y, d.z / e.z);
    for (uint32_t tier = 0; tier < 6u; tier++) {
        real t = (real)tier;
        real base = -0.6f + t * 0.27f;
        real height = minf_(0.66f - t * 0.045f, 1.0f - base);
        real radius = 0.94f - t * 0.148f;
        real ox = sin_d(t * 4.1f) * 0.022f, oz = cos_d(t * 3.7f) * 0.022f;
        v3 q = vsub(o, V(ox, base + height, oz));
        real k = radius / height;
        real a = v.x * v.x + v.z * v.z - k * k * v.y * v.y;
        real b = q.x * v.x + q.z * v.z - k * k * q.y * v.y;
        real c = q.x * q.x + q.z * q.z - k * k * q.y * q.y;
        real disc = b * b - a * c;
        if (r_fabs(a) < 1.0e-12f || disc < 0.0f) continue;
        for (uint32_t side = 0; side < 2u; side++) {
            real distance = (-b + (side == 1u ? r_sqrt(disc) : -r_sqrt(disc))) / a;
            v3 h = vadd(q, vmul(v, distance));
            if (distance <= 0.001f || distance >= result.t || h.y > 0.0f || h.y < -height) continue;
            real angle = atan2_d(h.z, h.x);
            real skirt = -h.y / height;
            real branches = 0.5f + 0.5f * sin_d(angle * (9.0f + t) + t * 3.7f);
            real needle = vnoise(vadds(vmulv(vadd(p, vmul(d, distance)), V(9.0f, 17.0f, 9.0f)), t * 7.0f));
            if (skirt > 0.76f + 0.19f * branches || (skirt > 0.4f && needle < 0.26f)) continue;
            result.n = vnormalize(V(h.x / e.x, -k * k * h.y / e.y, h.z / e.z));
            result.t = distance;
        }
    }
    return result;
}
static veg_hit grass_hit(v3 p, v3 d, v3 e) {
    veg_hit result = {V(0.0f, 0.0f, 0.0f), 1.0e30f};
    for (uint32_t blade = 0; blade < 9u; blade++) {
        real i = (real)blade;
        real angle = i * 2.39996f;
        v3 side = V(cos_d(angle), 0.0f, sin_d(angle));
        v3 base = vsub(vmul(vmul(side, e.x), 0.15f), V(0.0f, e.y, 0.0f));
        v3 tip = vadd(vmul(vmul(side, e.x), 0.6f + 0.3f * sin_d(i * 3.0f)),
                      V(0.0f, e.y * (0.5f + 0.5f * cos_d(i * 1.3f)), 0.0f));
        v3 width = vmul(V(-side.z, 0.0f, side.x), 0.035f);
        v3 hit = t_triangle(p, d, vsub(base, width), vadd(base, width), tip);
        if (hit.z < result.t) {
            v3 normal = vnormalize(vcross(width, vsub(tip, base)));
            if (vdot(normal, d) > 0.0f) normal = vneg(normal);
            result.n = normal;
            result.t = hit.z;
        }
    }
    return result;
}
/* The vegetation branch of landscape_query (ground.wgsl:197-202). */
static veg_hit vegetation_hit(real kind, v3 p, v3 d, v3 e) {
    if (kind < 3.5f) return conifer_hit(p, d, e);
    if (kind < 4.5f) return grass_hit(p, d, e);
    return trunk_hit(p, d, e);
}

/* landscape_query: ground.wgsl:123-242 */
static hit_t landscape_query(const scene *S, ray_t ray, real limit, int occlusion) {
    hit_t closest = {limit, MISS, {0, 0, 0}};
    if (S->s->g.ground_north[3] == 0.0f) return closest;
    v3 o = ground_origin(S, ray);
    v3 d = to_ground(S, ray.dir);
    real radius = S->s->g.ground_up[3];
    if (vdot(o, o) > 4.0f * radius * radius) return sphere_hit(S, ray, (uint32_t)S->s->g.ground_north[3] - 1u);
    if (d.y >= 0.0f && o.y > landscape_top(S)) return closest;
    real a = vdot(d, d);
    real b = -radius * d.y - vdot(o, d);
    real c = (o.x * o.x + o.z * o.z) + o.y * (2.0f * radius + o.y);
    real h = b * b - a * c;
    if (h >= 0.0f) {
        real root = r_sqrt(h);
        real q = b + (b >= 0.0f ? root : -root);
        if (q != 0.0f) {
            real t0 = minf_(c / q, q / a);
            real t1 = maxf_(c / q, q / a);
            real distance = t0 > 0.001f ? t0 : t1;
            if (distance > 0.001f && distance / METRES_PER_AU < closest.distance) {
                if (occlusion) { hit_t r = {distance / METRES_PER_AU, LOCAL_BASE, {0, 0, 0}}; return r; }
                v3 p = vadd(o, vmul(d, distance));
                v3 n = vnormalize(V(p.x / radius, 1.0f + p.y / radius, p.z / radius));
                closest.distance = distance / METRES_PER_AU;
                closest.index = LOCAL_BASE;
                closest.normal = from_ground(S, n);
            }
        }
    }
    if (S->s->g.ground_counts[1] != 0u && S->t && S->t->terrain) {
        real tl = minf_(closest.distance, 1.0e18f) * METRES_PER_AU;
        v3 tn = V(0, 0, 0);
        real tt = t_query(S, S->t->terrain, t_cells(S), o, d, tl, occlusion, &tn);
        if (tt < tl && tt < 1.0e29f) {
            closest.distance = tt / METRES_PER_AU;
            closest.index = TERRAIN_ID;
            closest.normal = from_ground(S, tn);
            if (occlusion) return closest;
        }
    }
    const sg_primitive *objects = S->t ? S->t->ground : NULL;
    uint32_t n_objects = S->s->g.ground_counts[0];
    for (uint32_t i = 0; objects && i < n_objects; i++) {
        const sg_primitive *object = &objects[i];
        v3 center = V(object->center[0], object->center[1], object->center[2]);
        v3 e = V(object->extent[0], object->extent[1], object->extent[2]);
        real kind = object->center[3];
        if (kind < 0.0f) {
            EV(prop_boxes);
            real bn, bf_;
            box_interval(vsub(o, center), d, e, &bn, &bf_);
            if (bn > bf_ || bf_ <= 0.001f || bn / METRES_PER_AU > closest.distance) i += (uint32_t)(-kind);
            continue;
        }
        EV(prop_tests);
        v3 p = vsub(o, center), v = d;
        v3 angles = V(0, 0, 0);
        if (kind == 2.25f) {
            angles = rock_angles(object->extent[3]);
            p = rock_to_local(p, angles);
            v = rock_to_local(v, angles);
        } else {
            p = rotate_north(p, -object->extent[3]);
            v = rotate_north(v, -object->extent[3]);
        }
        real distance = 1.0e30f;
        v3 n = V(0, 0, 0);
        if (kind > 2.5f) {
            real bn, bf_;
            box_interval(p, v, e, &bn, &bf_);
            if (bn > bf_ || bf_ <= 0.001f || bn / METRES_PER_AU > closest.distance) continue;
            veg_hit vegetation = vegetation_hit(kind, p, v, e);
            distance = vegetation.t;
            n = vegetation.n;
        } else if (kind > 1.5f) {
            real bn, bf_;
            box_interval(p, v, e, &bn, &bf_);
            if (bn > bf_ || bf_ <= 0.001f || bn / METRES_PER_AU > closest.distance) continue;
            distance = rock_hit(p, v, e, &n);
        } else if (kind > 0.5f) {
            v3 sp = V(p.x / e.x, p.y / e.y, p.z / e.z);
            v3 sd = V(v.x / e.x, v.y / e.y, v.z / e.z);
            real aa = vdot(sd, sd), bb = vdot(sp, sd), cc = vdot(sp, sp) - 1.0f;
            real hh = bb * bb - aa * cc;
            if (hh >= 0.0f) {
                real root = r_sqrt(hh);
                distance = (-bb - root) / aa;
                if (distance <= 0.001f) distance = (-bb + root) / aa;
                v3 hp = vadd(p, vmul(v, distance));
                n = vnormalize(V(hp.x / (e.x * e.x), hp.y / (e.y * e.y), hp.z / (e.z * e.z)));
            }
        } else {
            real in_, out_;
            box_interval(p, v, e, &in_, &out_);
            if (in_ <= out_ && out_ > 0.001f) {
                distance = in_ > 0.001f ? in_ : out_;
                v3 hp = vadd(p, vmul(v, distance));
                v3 point = V(hp.x / e.x, hp.y / e.y, hp.z / e.z);
                v3 ap = V(r_fabs(point.x), r_fabs(point.y), r_fabs(point.z));
                real sx = point.x > 0 ? 1.0f : (point.x < 0 ? -1.0f : 0.0f);
                real sy = point.y > 0 ? 1.0f : (point.y < 0 ? -1.0f : 0.0f);
                real sz = point.z > 0 ? 1.0f : (point.z < 0 ? -1.0f : 0.0f);
                if (ap.x >= ap.y && ap.x >= ap.z) n.x = sx;
                else if (ap.y >= ap.z) n.y = sy;
                else n.z = sz;
            }
        }
        if (distance > 0.001f && distance < 1.0e29f && distance / METRES_PER_AU < closest.distance) {
            if (occlusion) { hit_t r = {distance / METRES_PER_AU, LOCAL_BASE + 1u + i, {0, 0, 0}}; return r; }
            if (kind == 2.25f) n = rock_from_local(n, angles);
            else n = rotate_north(n, object->extent[3]);
            closest.distance = distance / METRES_PER_AU;
            closest.index = LOCAL_BASE + 1u + i;
            closest.normal = from_ground(S, n);
        }
    }
    return closest;
}

/* landscape_point: ground.wgsl:252-254 */
static v3 landscape_point(const scene *S, ray_t ray, hit_t hit) {
    return vadd(ground_origin(S, ray), vmul(to_ground(S, ray.dir), hit.distance * METRES_PER_AU));
}

static real smooth_footprint(const scene *S, real distance) {
    return distance * 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
}

/* forest_floor, desert_floor, crater_floor: ground.wgsl:256-317 */
static v3 v3mix(v3 a, v3 b, real t) { return V(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t)); }
static v3 forest_floor(const scene *S, v3 p, real distance, v3 normal) {
    real broad = vnoise(vadd(vmul(p, 0.045f), V(7.0f, 0.0f, 13.0f)));
    real middle = vnoise(vmul(p, 0.7f));
    real grain = vnoise(vmul(p, 18.0f));
    real footprint = smooth_footprint(S, distance);
    real detail = 1.0f - smoothstepf(0.006f, 0.055f, footprint);
    v3 moss = v3mix(V(0.028f, 0.054f, 0.014f), V(0.105f, 0.14f, 0.039f), middle);
    v3 earth = v3mix(V(0.055f, 0.029f, 0.013f), V(0.17f, 0.115f, 0.057f), middle);
    v3 color = v3mix(earth, moss, smoothstepf(0.35f, 0.63f, broad));
    real needles = r_pow(maxf_(0.0f, r_sin(p.x * 92.0f + p.z * 137.0f + middle * 7.0f)), 18.0f) *
                    smoothstepf(0.50f, 0.68f, grain);
    color = v3mix(color, V(0.22f, 0.145f, 0.067f), needles * detail * 0.5f);
    color = vmul(color, 1.0f + (grain - 0.5f) * 0.38f * detail);
    real slope = 1.0f - maxf_(normal.y, 0.0f);
    v3 stone = v3mix(V(0.095f, 0.105f, 0.10f), V(0.24f, 0.23f, 0.20f), middle);
    color = v3mix(color, stone, smoothstepf(0.10f, 0.43f, slope + (broad - 0.5f) * 0.17f));
    real center = 2.0f + 0.30f * p.z + 2.0f * r_sin(p.z * 0.055f);
    real edge = r_fabs(p.x - center) + (middle - 0.5f) * 0.55f;
    real path = (1.0f - smoothstepf(0.8f, 2.1f, edge)) * (1.0f - smoothstepf(45.0f, 95.0f, p.z)) *
                 smoothstepf(-10.0f, 0.0f, p.z);
    v3 gravel = v3mix(V(0.12f, 0.095f, 0.062f), V(0.26f, 0.23f, 0.17f), grain * detail + 0.5f * (1.0f - detail));
    return v3mix(color, gravel, path * 0.85f);
}
static v3 desert_floor(const scene *S, v3 p, real distance, v3 normal) {
    real broad = vnoise(vadd(vmul(p, 0.007f), V(19.0f, 2.0f, 4.0f)));
    real gravel = vnoise(vmul(p, 2.8f));
    real footprint = smooth_footprint(S, distance);
    real detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    v3 sand = v3mix(V(0.31f, 0.21f, 0.125f), V(0.53f, 0.40f, 0.26f), broad);
    v3 rock = v3mix(V(0.18f, 0.10f, 0.055f), V(0.38f, 0.245f, 0.145f), broad);
    v3 color = v3mix(sand, rock, smoothstepf(0.08f, 0.4f, 1.0f - maxf_(normal.y, 0.0f)));
    color = vmul(color, 1.0f + (gravel - 0.5f) * 0.32f * detail);
    real center = 2.8f + 0.55f * r_sin(p.z / 38.0f) + 1.4f * r_sin(p.z / 210.0f);
    real edge = r_fabs(p.x - center);
    real aa = maxf_(0.015f, footprint * 0.5f);
    real fade = (1.0f - smoothstepf(0.25f, 0.9f, footprint)) * (1.0f - smoothstepf(1000.0f, 2200.0f, r_fabs(p.z))) *
                 (1.0f - smoothstepf(0.12f, 0.35f, 1.0f - maxf_(normal.y, 0.0f)));
    real worn = 1.0f - smoothstepf(0.8f, 1.2f, edge);
    real rut_edge = r_fabs(edge - 0.68f) + (gravel - 0.5f) * 0.1f * detail;
    real tracks = 1.0f - smoothstepf(0.12f - aa, 0.23f + aa, rut_edge);
    v3 packed = vmul(sand, 0.72f + 0.10f * gravel * detail);
    color = v3mix(color, vmul(sand, 0.93f), worn * fade * 0.35f);
    return v3mix(color, packed, tracks * fade * 0.8f);
}
static v3 crater_floor(const scene *S, v3 p, real distance, v3 normal) {
    real broad = vnoise(vadd(vmul(p, 0.004f), V(3.0f, 0.0f, 8.0f)));
    real middle = vnoise(vmul(p, 0.09f));
    real grain = vnoise(vmul(p, 3.1f));
    real footprint = smooth_footprint(S, distance);
    real detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    real tone = mixf(0.11f, 0.21f, broad) * (0.86f + 0.28f * middle);
    tone *= 1.0f + 0.35f * smoothstepf(0.15f, 0.5f, 1.0f - maxf_(normal.y, 0.0f));
    tone *= 1.0f + (grain - 0.5f) * 0.3f * detail;
    return V(tone, tone * 0.97f, tone * 0.93f);
}

/* Albedo-map extension: nearest texel at surface-frame (x, z). */
static size_t map_texel(const scene *S, v3 p) {
    const oracle_tables *t = S->t;
    real u = (p.x / t->map_extent + 1.0f) * 0.5f * (real)t->map_width;
    real w = (p.z / t->map_extent + 1.0f) * 0.5f * (real)t->map_height;
    int32_t i = (int32_t)r_floor(u), j = (int32_t)r_floor(w);
    if (i < 0) i = 0;
    if (j < 0) j = 0;
    if (i > (int32_t)t->map_width - 1) i = (int32_t)t->map_width - 1;
    if (j > (int32_t)t->map_height - 1) j = (int32_t)t->map_height - 1;
    return (size_t)j * t->map_width + (size_t)i;
}
static real map_albedo(const scene *S, v3 p) { return S->t->albedo_map[map_texel(S, p)]; }

/* landscape_albedo: ground.wgsl:597-632 (themes 0-2; vegetation kinds are
 * rejected), with the albedo-map extension for the ground itself. */
/* ---------------------------------------------------------------- */
/* Landscape themes 3 (alpine) and 5 (dunes): ground.wgsl:320-596,   */
/* terrain.wgsl:142-150. Strict f32 with correctly rounded            */
/* transcendentals, like the surface styles.                          */
/* ---------------------------------------------------------------- */
#define ICE_FLOW 4.4f
#define DUNE_WIND 0.61f
#define DUNE_PAN_LEVEL 2.0f
typedef struct { real x, y; } v2;
static inline v2 V2(real x, real y) { v2 r = {x, y}; return r; }
static inline real v2dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline real v2len(v2 a) { return r_sqrt(a.x * a.x + a.y * a.y); }

static inline real terrain_scale(const scene *S) { return clampf_(S->s->g.ground_up[3] / 200000.0f, 0.0001f, 1.0f); }
static inline real footprint_at(const scene *S, real distance) {
    return distance * 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
}
/* The surface-frame point in terrain units above the curved datum. */
static inline v3 terrain_local(const scene *S, v3 p) {
    real c = t_curvature(p.x, p.z, S->s->g.ground_up[3]);
    return vdivs(V(p.x, p.y - c, p.z), terrain_scale(S));
}

/* lookout_hill: ground.wgsl:322-325 */
static real lookout_hill(real r) {
    real u = minf_(v2len(V2(r, 30.0f)) / 700.0f, 1.0f);
    return 180.0f * (1.0f - u) * (1.0f - u);
}

/* dune_cracks: ground.wgsl:490-503 (the gap between the two nearest
 * jittered cells). */
static real dune_cracks(v2 p) {
    v2 g = V2(r_floor(p.x), r_floor(p.y));
    v2 f = V2(p.x - g.x, p.y - g.y);
    real d1 = 8.0f, d2 = 8.0f;
    for (int j = -1; j <= 1; j++) {
        for (int i = -1; i <= 1; i++) {
            v2 o = V2((real)i, (real)j);
            v3 h = hash33(V(g.x + o.x, g.y + o.y, 3.0f));
            real d = v2len(V2(o.x + 0.15f + 0.7f * h.x - f.x, o.y + 0.15f + 0.7f * h.y - f.y));
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
static v2 ice_crevasse(v2 q, real footprint) {
    real r = v2len(q);
    real tension = smoothstepf(650.0f, 900.0f, r) * (1.0f - smoothstepf(1800.0f, 2600.0f, r));
    real strain = maxf_(smoothstepf(0.47f, 0.58f, fbm(V(q.x / 2600.0f + 4.0f, 2.0f, q.y / 2600.0f), 2)), tension) *
                   smoothstepf(600.0f, 750.0f, r);
    if (strain <= 0.0f) return V2(0.0f, 0.0f);
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    real along = v2dot(q, flow) + 280.0f * (vnoise(V(q.x / 1500.0f, q.y / 1500.0f, 1.0f)) - 0.5f);
    real across = v2dot(q, V2(flow.y, -flow.x)) + 120.0f * (vnoise(V(q.x / 900.0f, q.y / 900.0f, 5.0f)) - 0.5f);
    real spacing = 60.0f;
    real row = r_floor(along / spacing);
    uint32_t key = hash_u32(((uint32_t)(int32_t)row * 0x8da6b343u) ^ 0xc3e5u);
    real length_m = 120.0f + 300.0f * (real)(key & 255u) / 255.0f;
    real s = across / length_m + (real)((key >> 8u) & 255u) / 255.0f;
    real segment = r_floor(s);
    real lens = pow_d(maxf_(sin_d(PI_F * (s - segment)), 0.0f), 0.7f);
    uint32_t open = hash_u32(key ^ (uint32_t)(int32_t)segment);
    if ((open & 255u) < 70u) return V2(0.0f, 0.0f);
    real centre = 0.5f + 0.3f * ((real)((open >> 8u) & 255u) / 255.0f - 0.5f);
    real half_width = 0.5f * (2.0f + 14.0f * (real)((open >> 16u) & 255u) / 255.0f) * lens * strain;
    real d = r_fabs(along / spacing - row - centre) * spacing + 0.8f * (vnoise(V(q.x * 0.15f, q.y * 0.15f, 9.0f)) - 0.5f);
    real aa = maxf_(footprint, 1.0e-3f);
    real coverage = clampf_((half_width - d) / aa + 0.5f, 0.0f, 1.0f) * minf_(1.0f, 2.0f * half_width / aa);
    return V2(coverage, 1.0f - clampf_(d / maxf_(half_width, 1.0e-3f), 0.0f, 1.0f));
}

/* alpine_floor: ground.wgsl:365-427 */
static v3 alpine_floor(const scene *S, v3 p, real distance, v3 normal) {
    real scale = terrain_scale(S);
    v3 q = terrain_local(S, p);
    real hill = lookout_hill(v2len(V2(q.x, q.z)));
    q.y = q.y - hill;
    real footprint = footprint_at(S, distance) / scale;
    real detail = 1.0f - smoothstepf(0.025f, 0.2f, footprint);
    real slope = 1.0f - maxf_(normal.y, 0.0f);
    real broad = vnoise(vadd(vmul(q, 0.004f), V(11.0f, 4.0f, 1.0f)));
    real middle = vnoise(vmul(q, 0.2f));
    real grain = vnoise(vmul(q, 4.0f));
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    real along = v2dot(V2(q.x, q.z), flow);
    real across = v2dot(V2(q.x, q.z), V2(flow.y, -flow.x));
    real crust = smoothstepf(0.45f, 0.6f, fbm(V(along * 0.004f, 2.0f, across * 0.012f), 3));
    v3 snow = vmix(V(0.86f, 0.88f, 0.91f), V(0.76f, 0.8f, 0.86f), crust);
    snow = vmul(snow, 0.97f + 0.05f * middle);
    real bare = smoothstepf(0.47f, 0.53f, fbm(vadd(vmul(q, 0.0016f), V(3.0f, 0.0f, 8.0f)), 4) + 0.1f * (broad - 0.5f));
    v3 ice = vmix(V(0.36f, 0.55f, 0.7f), V(0.52f, 0.67f, 0.78f), middle);
    real fracture_width = 0.03f + footprint / 4.0f;
    real fractures = (1.0f - smoothstepf(0.0f, fracture_width, dune_cracks(V2(q.x / 4.0f + 9.0f, q.z / 4.0f + 9.0f)))) *
                      0.03f / fracture_width;
    ice = vmix(ice, V(0.82f, 0.86f, 0.9f), minf_(fractures, 1.0f) * 0.7f);
    ice = vmul(ice, 1.0f + (grain - 0.5f) * 0.12f * detail);
    v3 glacier = vmix(snow, ice, bare);
    v3 debris = vmix(V(0.12f, 0.115f, 0.11f), V(0.26f, 0.24f, 0.22f), grain);
    real dirty = smoothstepf(6.0f, 30.0f, q.y) * (1.0f - smoothstepf(30.0f, 70.0f, q.y));
    glacier = vmix(glacier, vmix(debris, glacier, 0.45f), dirty * smoothstepf(0.4f, 0.7f, broad) * 0.8f);
    real wall = smoothstepf(0.35f, 0.6f, slope) * (1.0f - smoothstepf(20.0f, 45.0f, q.y));
    real depth = smoothstepf(4.0f, -4.0f, q.y);
    v3 blue = vmix(V(0.32f, 0.55f, 0.72f), V(0.1f, 0.25f, 0.42f), depth);
    glacier = vmix(glacier, vmul(blue, 0.9f + 0.2f * middle), wall);
    v2 crack = ice_crevasse(V2(q.x, q.z), footprint);
    real fade = 1.0f - smoothstepf(10.0f, 25.0f, q.y);
    crack = V2(crack.x * fade, crack.y * fade);
    real lip = (1.0f - smoothstepf(0.0f, 0.12f, crack.y)) * crack.x;
    v3 inside = vmix(V(0.3f, 0.55f, 0.74f), V(0.02f, 0.06f, 0.12f), smoothstepf(0.1f, 0.8f, crack.y));
    glacier = vmix(glacier, inside, crack.x);
    glacier = vmix(glacier, V(0.9f, 0.92f, 0.95f), lip * 0.5f);
    real mountain = maxf_(smoothstepf(25.0f, 70.0f, q.y + 30.0f * (broad - 0.5f)), smoothstepf(4.0f, 15.0f, hill));
    real joints = 1.0f - smoothstepf(0.0f, 0.06f + footprint / 3.0f,
                                      dune_cracks(V2((q.x + q.y * 0.5f) / 3.0f, q.z / 3.0f)));
    v3 granite = vmix(V(0.09f, 0.085f, 0.08f), V(0.24f, 0.215f, 0.19f), broad);
    granite = vmul(granite, 0.85f + 0.3f * middle - 0.35f * joints * (1.0f - smoothstepf(0.1f, 1.0f, footprint)));
    real lichen = smoothstepf(0.68f, 0.78f, vnoise(vmul(q, 0.9f))) * (1.0f - smoothstepf(0.6f, 0.9f, slope));
    granite = vmix(granite, V(0.3f, 0.17f, 0.06f), lichen * 0.5f * detail);
    real cover = 1.0f - smoothstepf(0.17f, 0.33f, slope + (broad - 0.5f) * 0.18f + (middle - 0.5f) * 0.08f);
    real scoured = smoothstepf(0.52f, 0.62f, fbm(vadd(vmul(q, 0.012f), V(2.0f, 0.0f, 6.0f)), 4)) *
                    smoothstepf(25.0f, 90.0f, hill) * (1.0f - smoothstepf(150.0f, 172.0f, hill));
    real cover_hill = cover * (1.0f - scoured);
    v3 peak = vmix(granite, snow, cover_hill);
    v3 color = vmix(glacier, peak, mountain);
    return vmul(color, 1.0f + (grain - 0.5f) * 0.08f * detail);
}

/* alpine_shading_normal: ground.wgsl:430-459 (telescope-space normal in
 * and out, surface-frame point). */
static v3 alpine_shading_normal(const scene *S, v3 p, real distance, v3 normal) {
    real footprint = footprint_at(S, distance);
    v3 n = to_ground(S, normal);
    real snowy = 1.0f - smoothstepf(0.3f, 0.5f, 1.0f - n.y);
    v2 flow = V2(sin_d(ICE_FLOW), cos_d(ICE_FLOW));
    v2 side = V2(flow.y, -flow.x);
    v2 gradient = V2(0.0f, 0.0f);
    real scale = 1.2f, strength = 0.2f;
    for (uint32_t octave = 0; octave < 3u; octave++) {
        real fade = 1.0f - smoothstepf(0.08f * scale, 0.25f * scale, footprint);
        if (fade > 0.0f) {
            real a = v2dot(V2(p.x, p.z), flow) / (6.0f * scale);
            real c = v2dot(V2(p.x, p.z), side) / scale;
            real e = 0.08f;
            real o = (real)octave * 13.0f;
            real da = vnoise(V(a + e, o, c)) - vnoise(V(a - e, o, c));
            real dc = vnoise(V(a, o, c + e)) - vnoise(V(a, o, c - e));
            real ridge_ = 1.0f + 1.5f * (1.0f - r_fabs(vnoise(V(a, o, c)) * 2.0f - 1.0f));
            real k = strength * fade * ridge_ * scale;
            real gx = (flow.x * da / (6.0f * scale) + side.x * dc / scale) / (2.0f * e) * k;
            real gz = (flow.y * da / (6.0f * scale) + side.y * dc / scale) / (2.0f * e) * k;
            gradient = V2(gradient.x + gx, gradient.y + gz);
        }
        scale *= 6.0f;
        strength *= 0.6f;
    }
    gradient = V2(gradient.x * snowy, gradient.y * snowy);
    return vnormalize(vadd(normal, from_ground(S, V(-gradient.x, 0.0f, -gradient.y))));
}

/* dune_pan: ground.wgsl:483-486 */
static v3 dune_pan(uint32_t i) {
    return i == 0u ? V(842.6f, 707.1f, 560.0f) : V(4346.7f, 1164.7f, 900.0f);
}

/* dune_floor: ground.wgsl:509-568 */
static v3 dune_floor(const scene *S, v3 p, real distance, v3 normal) {
    real scale = terrain_scale(S);
    v3 q = terrain_local(S, p);
    real footprint = footprint_at(S, distance) / scale;
    real detail = 1.0f - smoothstepf(0.02f, 0.15f, footprint);
    real slope = 1.0f - maxf_(normal.y, 0.0f);
    real broad = vnoise(vadd(vmul(q, 0.0015f), V(1.0f, 7.0f, 3.0f)));
    real middle = vnoise(vmul(q, 0.05f));
    real rise = smoothstepf(6.0f, 160.0f, q.y + 40.0f * (broad - 0.5f));
    v3 plinth = vmix(V(0.3f, 0.095f, 0.038f), V(0.36f, 0.12f, 0.045f), broad);
    v3 upper = vmix(V(0.42f, 0.155f, 0.06f), V(0.47f, 0.19f, 0.072f), broad);
    v3 sand = vmul(vmix(plinth, upper, rise), 0.94f + 0.08f * middle);
    real flat = v2len(V2(normal.x, normal.z));
    if (flat > 1.0e-3f) {
        v2 down = V2(-normal.x / flat, -normal.z / flat);
        real across = v2dot(V2(q.x, q.z), V2(-down.y, down.x));
        real along = v2dot(V2(q.x, q.z), down);
        real tongues = fbm(V(across * 0.18f, along * 0.012f, 5.0f), 3);
        real slip = smoothstepf(0.32f, 0.45f, slope);
        sand = vmix(sand, vmul(vmulv(sand, V(1.06f, 1.12f, 1.16f)), 0.86f + 0.28f * tongues), slip);
    }
    real lag = smoothstepf(0.6f, 0.76f, fbm(vadd(vmulv(q, V(0.013f, 0.0f, 0.004f)), V(9.0f, 0.0f, 2.0f)), 4)) *
                (1.0f - smoothstepf(0.04f, 0.16f, slope)) * (1.0f - smoothstepf(10.0f, 45.0f, q.y));
    sand = vmix(sand, V(0.13f, 0.065f, 0.05f), lag * 0.55f);
    real corridor = (1.0f - smoothstepf(5.0f, 16.0f, q.y + 6.0f * (broad - 0.5f))) *
                     (1.0f - smoothstepf(0.03f, 0.1f, slope));
    v3 gravel = vmix(V(0.39f, 0.21f, 0.115f), V(0.45f, 0.28f, 0.16f), vnoise(vmul(q, 0.3f)));
    real pebbles = smoothstepf(0.72f, 0.8f, vnoise(vmul(q, 7.0f))) * detail;
    sand = vmix(sand, vmul(gravel, 1.0f - 0.45f * pebbles), corridor * 0.6f);
    real pan = 0.0f;
    for (uint32_t i = 0; i < 2u; i++) {
        v3 c = dune_pan(i);
        pan = maxf_(pan, 1.0f - smoothstepf(c.z * 1.2f, c.z * 1.35f + 140.0f, v2len(V2(q.x - c.x, q.z - c.y))));
    }
    pan *= 1.0f - smoothstepf(DUNE_PAN_LEVEL + 0.25f, DUNE_PAN_LEVEL + 1.5f, q.y);
    if (pan > 0.0f) {
        real tone = fbm(vadd(vmul(q, 0.012f), V(4.0f, 0.0f, 1.0f)), 4);
        v3 clay = vmix(V(0.4f, 0.35f, 0.29f), V(0.6f, 0.56f, 0.49f), smoothstepf(0.3f, 0.7f, tone));
        clay = vmul(clay, 0.82f + 0.18f * smoothstepf(0.35f, 1.0f, pan));
        real fine_width = 0.04f + footprint / 0.9f;
        real cracks = (1.0f - smoothstepf(0.0f, fine_width, dune_cracks(V2(q.x / 0.9f, q.z / 0.9f)))) * 0.04f / fine_width;
        real wide_width = 0.03f + footprint / 6.0f;
        real large = (1.0f - smoothstepf(0.0f, wide_width, dune_cracks(V2(q.x / 6.0f + 17.0f, q.z / 6.0f + 17.0f)))) *
                      0.03f / wide_width;
        clay = vmul(clay, 1.0f - 0.6f * minf_(cracks, 1.0f) - 0.45f * minf_(large, 1.0f));
        clay = vmul(clay, 0.92f + 0.16f * vnoise(vmul(q, 2.3f)) * (1.0f - smoothstepf(0.04f, 0.25f, footprint)));
        sand = vmix(sand, clay, pan);
    }
    return vmul(sand, 1.0f + (vnoise(vmul(q, 9.0f)) - 0.5f) * 0.12f * detail);
}

/* dune_ripples: ground.wgsl:571-582; the surface-frame (x, z) gradient. */
static v2 dune_ripples(v3 p, real wavelength, real warp, real amplitude) {
    v2 wind = V2(sin_d(DUNE_WIND), cos_d(DUNE_WIND));
    v2 side = V2(wind.y, -wind.x);
    real bend = warp * (vnoise(V(p.x / (9.0f * wavelength), p.z / (9.0f * wavelength), 1.0f)) +
                         0.35f * vnoise(V(p.x / (2.5f * wavelength), p.z / (2.5f * wavelength), 7.0f)));
    real phase = v2dot(V2(p.x, p.z), wind) / wavelength + bend +
                  0.4f * sin_d(v2dot(V2(p.x, p.z), side) / (3.0f * wavelength));
    real theta = TAU_F * phase;
    real slope = cos_d(theta + 0.65f * sin_d(theta)) * (1.0f + 0.65f * cos_d(theta));
    real patches = smoothstepf(0.25f, 0.6f, vnoise(V(p.x / (14.0f * wavelength), p.z / (14.0f * wavelength), 3.0f)));
    real k = slope * amplitude * TAU_F / wavelength * patches;
    return V2(wind.x * k, wind.y * k);
}

/* dune_shading_normal: ground.wgsl:583-595 */
static v3 dune_shading_normal(const scene *S, v3 p, real distance, v3 normal) {
    real footprint = footprint_at(S, distance);
    v3 n = to_ground(S, normal);
    real gentle = 1.0f - smoothstepf(0.22f, 0.38f, 1.0f - n.y);
    v3 q = terrain_local(S, p);
    real dry = smoothstepf(DUNE_PAN_LEVEL + 0.4f, DUNE_PAN_LEVEL + 1.5f, q.y);
    v2 gradient = V2(0.0f, 0.0f);
    real fine = 1.0f - smoothstepf(0.03f, 0.07f, footprint);
    if (fine > 0.0f) {
        v2 r = dune_ripples(p, 0.12f, 2.5f, 0.006f);
        gradient = V2(gradient.x + r.x * fine, gradient.y + r.y * fine);
    }
    real coarse = (1.0f - smoothstepf(0.15f, 0.4f, footprint)) * (1.0f - smoothstepf(9.0f, 16.0f, q.y));
    if (coarse > 0.0f) {
        v2 r = dune_ripples(vadds(p, 31.0f), 0.8f, 2.0f, 0.03f);
        gradient = V2(gradient.x + r.x * coarse, gradient.y + r.y * coarse);
    }
    real k = gentle * dry;
    gradient = V2(gradient.x * k, gradient.y * k);
    return vnormalize(vadd(normal, from_ground(S, V(-gradient.x, 0.0f, -gradient.y))));
}

/* ---------------------------------------------------------------- */
/* Theme 4 (basalt): basalt_floor (ground.wgsl:463-477) and the      */
/* shading normals from the measured elevation atlas that follows the */
/* terrain's vertex cache (volcano.wgsl). Reads past the uploaded     */
/* atlas return 0 (the reference's buffer always holds one).          */
/* ---------------------------------------------------------------- */
static inline uint32_t u32_sat(real x) {
    if (!(x > 0.0f)) return 0u;
    if (x >= 4294967040.0f) return 0xffffffffu;
    return (uint32_t)x;
}
static inline int32_t i32_sat(real x) {
    if (!(x > -2147483520.0f)) return x != x ? 0 : (int32_t)0x80000000u;
    if (x >= 2147483520.0f) return 0x7fffffff;
    return (int32_t)x;
}
static inline real fract_(real x) { return x - r_floor(x); }
static inline real log2_d(real x) { return (real)log2((double)x); }
static real volcano_data(const scene *S, uint32_t i) {
    if (!S->t || !S->t->terrain || i >= S->t->terrain_detail_floats) return 0.0f;
    return S->t->terrain[oracle_terrain_floats(t_cells(S)) + i];
}
typedef struct { real x, y, z, w; } v4;
static v4 volcano_record(const scene *S, uint32_t i) {
    v4 r = {volcano_data(S, i), volcano_data(S, i + 1u), volcano_data(S, i + 2u), volcano_data(S, i + 3u)};
    return r;
}
static inline uint32_t clamp_index(int32_t v, uint32_t width) {
    int32_t hi = (int32_t)width - 1;
    return (uint32_t)(v < 0 ? 0 : (v > hi ? hi : v));
}
static real volcano_bilinear(const scene *S, uint32_t offset, uint32_t width, v2 uv) {
    v2 pixel = V2(uv.x * (real)width - 0.5f, uv.y * (real)width - 0.5f);
    int32_t lx = i32_sat(r_floor(pixel.x)), ly = i32_sat(r_floor(pixel.y));
    uint32_t ax = clamp_index(lx, width), ay = clamp_index(ly, width);
    uint32_t bx = clamp_index(lx == 0x7fffffff ? lx : lx + 1, width), by = clamp_index(ly == 0x7fffffff ? ly : ly + 1, width);
    v2 f = V2(fract_(pixel.x), fract_(pixel.y));
    return mixf(mixf(volcano_data(S, offset + ay * width + ax), volcano_data(S, offset + ay * width + bx), f.x),
                mixf(volcano_data(S, offset + by * width + ax), volcano_data(S, offset + by * width + bx), f.x), f.y);
}
static real volcano_map(const scene *S, uint32_t map, v2 p, real footprint) {
    v4 desc = volcano_record(S, map * 4u);
    v2 local = V2(p.x, p.y - desc.w);
    real reach = 0.5f * (desc.y - 1.0f) * desc.z;
    if (r_fabs(local.x) > reach || r_fabs(local.y) > reach) return 0.0f;
    v2 uv = V2((local.x / desc.z + 0.5f * desc.y) / desc.y, (local.y / desc.z + 0.5f * desc.y) / desc.y);
    real lod = maxf_(log2_d(maxf_(footprint / desc.z, 1.0f)), 0.0f);
    uint32_t offset = u32_sat(desc.x), width = u32_sat(desc.y);
    uint32_t levels = u32_sat(lod);
    for (uint32_t level = 0; level < levels && width > 1u; level++) {
        offset += width * width;
        width = (width + 1u) / 2u;
    }
    real a = volcano_bilinear(S, offset, width, uv);
    if (width == 1u) return a;
    real b = volcano_bilinear(S, offset + width * width, (width + 1u) / 2u, uv);
    return mixf(a, b, fract_(lod));
}
static real volcano_fine_weight(const scene *S, v2 p) {
    v4 desc = volcano_record(S, 4u);
    v2 local = V2(p.x, p.y - desc.w);
    real reach = 0.5f * (desc.y - 1.0f) * desc.z;
    return 1.0f - smoothstepf(reach - 72.0f, reach, maxf_(r_fabs(local.x), r_fabs(local.y)));
}
static real volcano_height(const scene *S, uint32_t map, v2 p, real footprint) {
    real coarse = volcano_map(S, map, p, footprint);
    if (map != 0u) return coarse;
    real weight = volcano_fine_weight(S, p);
    if (weight <= 0.0f) return coarse;
    return mixf(coarse, volcano_map(S, 1u, p, footprint), weight);
}
/* volcano_normal: volcano.wgsl:49-88 (surface-frame normals). */
static v3 volcano_normal(const scene *S, v3 p, real distance, v3 fallback) {
    real scale = terrain_scale(S);
    v2 point = V2(p.x / scale, p.z / scale);
    real footprint = footprint_at(S, distance) / scale;
    real best = 1.0f;
    uint32_t chosen = 0u;
    v2 local = V2(0.0f, 0.0f);
    v4 transform = {0.0f, 0.0f, 1.0f, 0.0f};
    real site_scale = 1.0f;
    for (uint32_t site = 0; site < 9u; site++) {
        v4 frame = volcano_record(S, 16u + site * 8u);
        v4 info = volcano_record(S, 20u + site * 8u);
        v2 relative = V2((point.x - frame.x) / info.x, (point.y - frame.y) / info.x);
        v2 q = V2(frame.z * relative.x - frame.w * relative.y, frame.w * relative.x + frame.z * relative.y);
        real height = volcano_height(S, u32_sat(info.y), q, footprint / info.x) * info.x;
        if (height > best) {
            best = height;
            chosen = u32_sat(info.y);
            local = q;
            transform = frame;
            site_scale = info.x;
        }
    }
    if (best <= 1.0f) return fallback;
    real spacing = volcano_record(S, chosen * 4u).z;
    if (chosen == 0u) spacing = mixf(spacing, 1.0f, volcano_fine_weight(S, local));
    real delta = maxf_(spacing, footprint / site_scale * 0.5f);
    real fp = footprint / site_scale;
    real dx = (volcano_height(S, chosen, V2(local.x + delta, local.y), fp) -
                volcano_height(S, chosen, V2(local.x - delta, local.y), fp)) / (2.0f * delta);
    real dz = (volcano_height(S, chosen, V2(local.x, local.y + delta), fp) -
                volcano_height(S, chosen, V2(local.x, local.y - delta), fp)) / (2.0f * delta);
    v2 gradient = V2(transform.z * dx + transform.w * dz, -transform.w * dx + transform.z * dz);
    real radius = S->s->g.ground_up[3];
    real k = r_sqrt(maxf_(radius * radius - (p.x * p.x + p.z * p.z), 1.0f));
    v2 curvature = V2(p.x / k, p.z / k);
    v3 n = vnormalize(V(-gradient.x + curvature.x, 1.0f, -gradient.y + curvature.y));
    if (vdot(n, fallback) < 0.2f) return vnormalize(vmix(fallback, n, 0.7f));
    return n;
}

/* basalt_floor: ground.wgsl:463-477 */
static v3 basalt_floor(const scene *S, v3 p, real distance, v3 normal) {
    real footprint = footprint_at(S, distance);
    real broad = fbm(vadd(vmul(p, 0.006f), V(5.0f, 9.0f, 2.0f)), 4);
    real weather = fbm(vadd(vmul(p, 0.017f), V(23.0f, 7.0f, 11.0f)), 3);
    real middle = mixf(fbm(vmul(p, 0.08f), 3), 0.5f, smoothstepf(1.0f, 12.0f, footprint));
    v3 ash = vmix(V(0.065f, 0.060f, 0.052f), V(0.14f, 0.12f, 0.095f), broad);
    v3 rock = vmix(V(0.028f, 0.030f, 0.031f), V(0.07f, 0.064f, 0.054f), middle);
    rock = vmix(rock, V(0.16f, 0.073f, 0.037f), smoothstepf(0.48f, 0.68f, weather) * 0.45f);
    real slope = 1.0f - maxf_(normal.y, 0.0f);
    real loose = 1.0f - smoothstepf(0.14f, 0.43f, slope + 0.12f * (weather - 0.5f));
    v3 color = vmix(rock, ash, loose);
    color = vmul(color, 0.86f + 0.28f * middle);
    real grain = vnoise(vmul(p, 5.0f));
    return vmul(color, 1.0f + (grain - 0.5f) * 0.28f * (1.0f - smoothstepf(0.025f, 0.2f, footprint)));
}

static v3 landscape_albedo(const scene *S, ray_t ray, hit_t hit) {
    v3 p = landscape_point(S, ray, hit);
    real distance = hit.distance * METRES_PER_AU;
    v3 n = to_ground(S, hit.normal);
    if (hit.index == LOCAL_BASE || hit.index == TERRAIN_ID) {
        if (S->t && S->t->albedo_map) { real a = map_albedo(S, p); return V(a, a, a); }
        switch (ground_theme(S)) {
            case 1u: return desert_floor(S, p, distance, n);
            case 2u: return crater_floor(S, p, distance, n);
            case 3u: return alpine_floor(S, p, distance, n);
            case 4u: return basalt_floor(S, p, distance, n);
            case 5u: return dune_floor(S, p, distance, n);
            default: return forest_floor(S, p, distance, n);
        }
    }
    const sg_primitive *object = &S->t->ground[hit.index - LOCAL_BASE - 1u];
    v3 tint = V(object->albedo[0], object->albedo[1], object->albedo[2]);
    real kind = object->albedo[3];
    if (kind == 0.0f) return tint;
    real middle = vnoise(vmul(p, 1.7f));
    real fine = mixf(vnoise(vmul(p, 12.0f)), 0.5f, smoothstepf(18.0f, 110.0f, distance));
    if (kind > 4.5f) return vmul(tint, 0.65f + 0.6f * middle);
    if (kind > 2.5f) {
        /* Conifers: bark on the lower trunk (ground.wgsl:618-625). */
        v3 q = rotate_north(vsub(p, V(object->center[0], object->center[1], object->center[2])), -object->extent[3]);
        q = V(q.x / object->extent[0], q.y / object->extent[1], q.z / object->extent[2]);
        if (kind > 3.5f || (q.y < -0.35f && r_sqrt(q.x * q.x + q.z * q.z) < 0.09f)) {
            real bark = vnoise(vmulv(p, V(25.0f, 1.5f, 25.0f)));
            return vmul(V(0.13f, 0.073f, 0.032f), 0.5f + 0.85f * bark);
        }
        return vmul(tint, 0.7f + 0.55f * middle + 0.2f * fine);
    }
    real strata = r_sin(p.y * 8.0f + 2.5f * middle);
    real lichen = smoothstepf(0.52f, 0.76f, middle) * maxf_(n.y, 0.0f);
    v3 stone = vmul(tint, 0.7f + 0.45f * fine + 0.07f * strata);
    if (ground_theme(S) != 0u) return stone;
    return v3mix(stone, V(0.11f, 0.145f, 0.037f), lichen * 0.65f);
}

/* Tangent of landscape_albedo: only the albedo-map texels are parameters. */
static v3 landscape_albedo_dot(const scene *S, const oracle_direction *D, ray_t ray, hit_t hit) {
    if (!D || !D->albedo_map || !S->t || !S->t->albedo_map) return V(0, 0, 0);
    if (hit.index != LOCAL_BASE && hit.index != TERRAIN_ID) return V(0, 0, 0);
    real d = D->albedo_map[map_texel(S, landscape_point(S, ray, hit))];
    return V(d, d, d);
}

/* landscape_shading_normal: ground.wgsl:633-648 (themes 0-2) */
static v3 landscape_shading_normal(const scene *S, ray_t ray, hit_t hit) {
    if (hit.index != LOCAL_BASE && hit.index != TERRAIN_ID) return hit.normal;
    v3 p = landscape_point(S, ray, hit);
    real distance = hit.distance * METRES_PER_AU;
    if (ground_theme(S) == 4u && hit.index == TERRAIN_ID)
        return from_ground(S, volcano_normal(S, p, distance, to_ground(S, hit.normal)));
    if (ground_theme(S) == 5u) return dune_shading_normal(S, p, distance, hit.normal);
    if (ground_theme(S) == 3u) return alpine_shading_normal(S, p, distance, hit.normal);
    real strength = 0.11f * (1.0f - smoothstepf(8.0f, 65.0f, distance));
    real dx = vnoise(vmul(vadd(p, V(0.025f, 0.0f, 0.0f)), 6.0f)) - vnoise(vmul(vsub(p, V(0.025f, 0.0f, 0.0f)), 6.0f));
    real dz = vnoise(vmul(vadd(p, V(0.0f, 0.0f, 0.025f)), 6.0f)) - vnoise(vmul(vsub(p, V(0.0f, 0.0f, 0.025f)), 6.0f));
    return vnormalize(vadd(hit.normal, vmul(from_ground(S, V(-dx, 0.0f, -dz)), strength)));
}

/* landscape_outgoing: ground.wgsl:649-662 */
static ray_t landscape_outgoing(const scene *S, ray_t ray, hit_t hit) {
    v3 p = landscape_point(S, ray, hit);
    if (hit.index == LOCAL_BASE) {
        real radius = S->s->g.ground_up[3];
        real d2 = p.x * p.x + p.z * p.z;
        if (p.y > -radius && d2 < radius * radius) p.y = -d2 / (radius + r_sqrt(radius * radius - d2));
    }
    p = vadd(p, vmul(to_ground(S, hit.normal), 0.005f));
    p.y -= S->s->g.ground_east[3];
    ray_t r;
    r.offset = vdivs(from_ground(S, p), METRES_PER_AU);
    r.dir = hit.normal;
    r.anchor = MISS;
    return r;
}

/* Russian roulette with survival s = clamp(max channel, 0.05, 0.95) of the
 * throughput t: its full tangent (t / s after survival) and the score of
 * the decision. The max channel is the first one reaching the maximum. */
static void roulette_tangent(v3 t, real s, int survived, v3 *dt_full, real *score) {
    real m = maxf_(t.x, maxf_(t.y, t.z));
    real dm = t.x >= m ? dt_full->x : (t.y >= m ? dt_full->y : dt_full->z);
    real ds = (m > 0.05f && m < 0.95f) ? dm : 0.0f;
    if (survived) {
        *score += ds / s;
        *dt_full = vdivs(vsub(*dt_full, vmul(vdivs(t, s), ds)), s);
    } else {
        *score += -ds / (1.0f - s);
    }
}

/* ---------------------------------------------------------------- */
/* Camera-only sky backdrop: pathtrace.wgsl:268-334                   */
/* ---------------------------------------------------------------- */
static v3 cam_right(const scene *S) { return V(S->s->g.cam_right[0], S->s->g.cam_right[1], S->s->g.cam_right[2]); }
static v3 cam_up(const scene *S) { return V(S->s->g.cam_up[0], S->s->g.cam_up[1], S->s->g.cam_up[2]); }
static v3 cam_fwd(const scene *S) { return V(S->s->g.cam_forward[0], S->s->g.cam_forward[1], S->s->g.cam_forward[2]); }

/* world_direction: :268-271 */
static v3 world_direction(const scene *S, v3 d) {
    return vnormalize(vsub(vadd(vmul(cam_right(S), d.x), vmul(cam_up(S), d.y)), vmul(cam_fwd(S), d.z)));
}

/* inside_star_dot: :118-128 */
static int inside_star_dot(const scene *S, v3 view, v3 star) {
    v3 sv = V(vdot(star, cam_right(S)), vdot(star, cam_up(S)), -vdot(star, cam_fwd(S)));
    if (sv.z >= 0.0f) return 0;
    real dx = view.x / -view.z - sv.x / -sv.z, dy = view.y / -view.z - sv.y / -sv.z;
    real scale = S->s->g.viewport[1] / (2.0f * S->s->g.cam_forward[3]);
    real px = dx * scale, py = dy * scale;
    return px * px + py * py <= STAR_DOT_PIXELS * STAR_DOT_PIXELS;
}

/* environment: :273-300 (primary rays only) */
static v3 environment(const scene *S, v3 view) {
    v3 light = V(0, 0, 0);
    const oracle_tables *t = S->t;
    if (!t || !t->catalogue || t->catalogue_n == 0u) return light;
    v3 dir = world_direction(S, view);
    real phi = r_atan2(dir.y, dir.x) + PI_F;
    real theta = r_acos(clampf_(dir.z, -1.0f, 1.0f));
    uint32_t x = (uint32_t)(phi * (256.0f / TAU_F));
    uint32_t y = (uint32_t)(theta * (128.0f / PI_F));
    if (x > 255u) x = 255u;
    if (y > 127u) y = 127u;
    uint32_t cell = y * 256u + x;
    for (uint32_t j = t->sky_cells[cell]; j < t->sky_cells[cell + 1u]; j++) {
        const float *star = t->catalogue + 8u * t->sky_cells[32769u + j];
        v3 sdir = V(star[0], star[1], star[2]);
        v3 perp = vcross(dir, sdir);
        if (vdot(dir, sdir) > 0.0f && vdot(perp, perp) <= star[3] && inside_star_dot(S, view, sdir))
            light = vadd(light, V(star[4], star[5], star[6]));
    }
    return light;
}

/* milky_way_texel, milky_way: :302-334 */
static v3 milky_way_texel(const scene *S, int x, int y) {
    int w = (int)S->s->background[1], h = (int)S->s->background[2];
    x = (x + w) % w;
    y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
    uint32_t packed = S->t->milky_way[(uint32_t)(y * w + x)];
    return vdivs(V((real)(packed & 1023u), (real)((packed >> 10) & 1023u), (real)((packed >> 20) & 1023u)),
                 1023.0f);
}
static v3 milky_way(const scene *S, v3 view) {
    if (S->s->background[0] == 0.0f || !S->t || !S->t->milky_way) return V(0, 0, 0);
    v3 dir = world_direction(S, view);
    v3 pole = vnormalize(V(0.35f, 0.82f, 0.45f));
    real a = -1.0f / (1.0f + pole.z);
    v3 right = V(pole.x * pole.y * a, 1.0f + pole.y * pole.y * a, -pole.y);
    v3 forward = vcross(pole, right);
    real longitude = r_atan2(vdot(dir, forward), vdot(dir, right));
    real u = 0.5f - longitude / TAU_F;
    real v = r_acos(clampf_(vdot(dir, pole), -1.0f, 1.0f)) / PI_F;
    real px = u * S->s->background[1] - 0.5f, py = v * S->s->background[2] - 0.5f;
    int lx = (int)r_floor(px), ly = (int)r_floor(py);
    real wx = px - r_floor(px), wy = py - r_floor(py);
    v3 top = vadd(vmul(milky_way_texel(S, lx, ly), 1.0f - wx), vmul(milky_way_texel(S, lx + 1, ly), wx));
    v3 bot = vadd(vmul(milky_way_texel(S, lx, ly + 1), 1.0f - wx), vmul(milky_way_texel(S, lx + 1, ly + 1), wx));
    return vmul(vadd(vmul(top, 1.0f - wy), vmul(bot, wy)), S->s->background[0]);
}


/* ---------------------------------------------------------------- */
/* Host atmosphere: pathtrace.wgsl:927-1234 (single-scattering        */
/* Rayleigh + Mie, planetshine) and the surface sky cache,            */
/* terrain.wgsl:286-329.                                              */
/* ---------------------------------------------------------------- */
#define ATMO_VIEW_STEPS 8u
#define ATMO_SUN_STEPS 4u
#define SKY_TEXELS 128u

static inline int air_on(const scene *S) { return S->s->g.atmo_params[3] >= 0.5f; }
static inline v3 atmo_center(const scene *S) {
    return V(S->s->g.atmo_center[0], S->s->g.atmo_center[1], S->s->g.atmo_center[2]);
}
static inline real host_radius(const scene *S) { return S->s->g.atmo_center[3]; }
static inline real atmosphere_top(const scene *S) { return S->s->g.atmo_center[3] + S->s->g.atmo_params[2]; }
static inline real atmo_scale_height(const scene *S) { return S->s->g.atmo_params[1]; }
static inline v3 vexp_neg(v3 beta, real x) {
    return V(r_exp(-beta.x * x), r_exp(-beta.y * x), r_exp(-beta.z * x));
}
static inline v3 beta_extinction(const scene *S) {
    const float *r = S->s->g.atmo_rayleigh;
    return V(r[0] + r[3], r[1] + r[3], r[2] + r[3]);
}
/* u32(ceil(x)) clamped to [2, ATMO_VIEW_STEPS] (the WGSL conversion
 * saturates; C's is undefined out of range). */
static inline uint32_t view_steps(real x) {
    real q = r_ceil(x);
    if (!(q > 2.0f)) return 2u;
    if (q >= (real)ATMO_VIEW_STEPS) return ATMO_VIEW_STEPS;
    return (uint32_t)q;
}

/* shell_exit: pathtrace.wgsl:945-956 */
static real shell_exit(const scene *S, v3 origin, v3 dir) {
    v3 oc = vsub(origin, atmo_center(S));
    real b = vdot(oc, dir);
    real top = atmosphere_top(S);
    real c = vdot(oc, oc) - top * top;
    real disc = b * b - c;
    if (disc < 0.0f) return 0.0f;
    return -b + r_sqrt(disc);
}

/* density_integral: pathtrace.wgsl:959-974 */
static real density_integral(const scene *S, v3 origin, v3 dir, uint32_t steps) {
    real distance = shell_exit(S, origin, dir);
    if (distance <= 0.0f) return 0.0f;
    real dt = distance / (real)steps;
    real inv_h = 1.0f / atmo_scale_height(S);
    real r = host_radius(S);
    real sum = 0.0f;
    for (uint32_t i = 0; i < steps; i++) {
        v3 p = vadd(origin, vmul(dir, ((real)i + 0.5f) * dt));
        real h = maxf_(vlength(vsub(p, atmo_center(S))) - r, 0.0f);
        sum += r_exp(-h * inv_h);
    }
    return sum * dt;
}

/* host_offset, inside_air, air_transmittance: pathtrace.wgsl:976-1002 */
static v3 host_offset(const scene *S, ray_t origin) {
    if (origin.anchor == MISS) return vsub(origin.offset, atmo_center(S));
    return vadd(vadd(vsub(b_center(S, origin.anchor), atmo_center(S)), b_low(S, origin.anchor)), origin.offset);
}
static int inside_air(const scene *S, ray_t origin) {
    if (S->s->g.atmo_params[3] < 0.5f) return 0;
    v3 oc = host_offset(S, origin);
    real top = atmosphere_top(S);
    return vdot(oc, oc) < top * top;
}
static v3 air_transmittance(const scene *S, ray_t origin, v3 dir) {
    if (!inside_air(S, origin)) return V(1, 1, 1);
    v3 p = vadd(atmo_center(S), host_offset(S, origin));
    return vexp_neg(beta_extinction(S), density_integral(S, p, dir, ATMO_SUN_STEPS));
}

/* rayleigh_phase, mie_phase: pathtrace.wgsl:1004-1010 */
static inline real rayleigh_phase(real cos_theta) {
    return 3.0f / (16.0f * PI_F) * (1.0f + cos_theta * cos_theta);
}
static inline real mie_phase(real cos_theta, real g) {
    real g2 = g * g;
    return (1.0f - g2) / (4.0f * PI_F * r_pow(1.0f + g2 - 2.0f * g * cos_theta, 1.5f));
}
static v3 phase_weight(const scene *S, real cos_theta) {
    const float *r = S->s->g.atmo_rayleigh;
    real g = S->s->g.atmo_params[0];
    real rp = rayleigh_phase(cos_theta), mp = mie_phase(cos_theta, g);
    real m = r[3] * mp;
    return V(r[0] * rp + m, r[1] * rp + m, r[2] * rp + m);
}

/* sample_reflector: pathtrace.wgsl:1017-1044 */
typedef struct { uint32_t index; real inverse_probability; } reflector_t;
static reflector_t sample_reflector(const scene *S, v3 origin, uint32_t *rng) {
    ray_t ray = {origin, V(0.0f, 0.0f, -1.0f), MISS};
    uint32_t host = (uint32_t)S->s->g.atmo_params[3] - 1u;
    uint32_t selected = MISS;
    real selected_weight = 0.0f, total = 0.0f;
    for (uint32_t b = 0; b < S->s->counts[0]; b++) {
        if (b == host || b_emissive(S, b) > 0.5f) continue;
        v3 c = b_color(S, b);
        real weight = cone_width(S, ray, b) * maxf_(c.x, maxf_(c.y, c.z));
        if (weight <= 0.0f) continue;
        total += weight;
        if (rnd(S, rng) * total < weight) {
            selected = b;
            selected_weight = weight;
        }
    }
    reflector_t r = {selected, total / maxf_(selected_weight, 1.0e-30f)};
    return r;
}

/* reflected_radiance: pathtrace.wgsl:1049-1073 */
static v3 reflected_radiance(const scene *S, ray_t ray, uint32_t index, uint32_t *rng) {
    hit_t hit = sphere_hit(S, ray, index);
    if (hit.index == MISS) return V(0, 0, 0);
    v3 albedo = surface_albedo(S, index, hit.normal);
    ray_t outgoing = {vmul(hit.normal, S->b[index].radius * (1.0f + 2.0e-6f)), hit.normal, index};
    v3 radiance = V(0, 0, 0);
    for (uint32_t slot = 0; slot < light_count(S); slot++) {
        uint32_t s = light_index(S, slot);
        if (b_emissive(S, s) < 0.5f) continue;
        light_sample light = sample_light(S, outgoing, s, rng);
        real cosine = maxf_(vdot(hit.normal, light.dir), 0.0f);
        if (cosine > 0.0f) {
            outgoing.dir = light.dir;
            radiance = vadd(radiance, vmul(vmulv(albedo, b_color(S, s)),
                                           cosine * light_visibility(S, outgoing, s) / (PI_F * light.pdf)));
        }
    }
    return radiance;
}

/* ground_reflector_pdf: src/guided_ground.rs:21-37 */
static real ground_reflector_pdf(const scene *S, ray_t ray) {
    uint32_t host = (uint32_t)S->s->g.atmo_params[3] - 1u;
    real total = 0.0f, density = 0.0f;
    for (uint32_t b = 0; b < S->s->counts[0]; b++) {
        if (b == host || b_emissive(S, b) > 0.5f) continue;
        real width = cone_width(S, ray, b);
        v3 c = b_color(S, b);
        real weight = width * maxf_(c.x, maxf_(c.y, c.z));
        if (weight <= 0.0f) continue;
        total += weight;
        if (sphere_hit(S, ray, b).index != MISS) density += weight / (TAU_F * width);
    }
    return density / maxf_(total, 1.0e-30f);
}

/* brightest_risen_light: pathtrace.wgsl:1078-1089 */
static real brightest_risen_light(const scene *S, v3 origin) {
    ray_t ray = {origin, V(0.0f, 0.0f, -1.0f), MISS};
    v3 up = V(S->s->g.ground_up[0], S->s->g.ground_up[1], S->s->g.ground_up[2]);
    real brightest = 0.0f;
    for (uint32_t slot = 0; slot < light_count(S); slot++) {
        uint32_t b = light_index(S, slot);
        if (b_emissive(S, b) < 0.5f) continue;
        if (vdot(vnormalize(relative_center(S, ray, b)), up) <= 0.0f) continue;
        v3 c = b_color(S, b);
        brightest = maxf_(brightest, maxf_(c.x, maxf_(c.y, c.z)) * TAU_F * cone_width(S, ray, b));
    }
    return brightest;
}

/* eclipse_light_samples: pathtrace.wgsl:239-262 */
static uint32_t eclipse_light_samples(const scene *S, ray_t ray, uint32_t index) {
    if (S->s->counts[1] != 0u) return 1u;
    v3 source = relative_center(S, ray, index);
    real distance = vlength(source);
    v3 axis = vdivs(source, distance);
    real source_chord = r_sqrt(2.0f * cone_width(S, ray, index));
    for (uint32_t b = 0; b < S->s->counts[0]; b++) {
        if (b == index) continue;
        v3 offset = relative_center(S, ray, b);
        real d2 = vdot(offset, offset);
        real radius = S->b[b].radius;
        if (d2 <= radius * radius) continue;
        real d = r_sqrt(d2);
        if (d - radius >= distance + S->b[index].radius) continue;
        real sin2 = clampf_(radius * radius / d2, 0.0f, 1.0f);
        real limb_chord = r_sqrt(2.0f * sin2 / (1.0f + r_sqrt(1.0f - sin2)));
        real separation = vlength(vsub(axis, vdivs(offset, d)));
        if (separation < source_chord + limb_chord && separation + source_chord > limb_chord) return 4u;
    }
    return 1u;
}

/* air_light_visibility: rings.wgsl:121-141 */
static real air_light_visibility(const scene *S, ray_t ray, uint32_t light) {
    if (S->s->g.ground_north[3] == 0.0f || ground_origin(S, ray).y <= landscape_top(S))
        return light_visibility(S, ray, light);
    hit_t surface = sphere_hit(S, ray, light);
    if (surface.index == MISS) return 0.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (i == light) continue;
        hit_t hit = sphere_hit(S, ray, i);
        if (hit.index != MISS && (hit.distance < surface.distance ||
                                  (hit.distance == surface.distance && i < light)))
            return 0.0f;
    }
    real transmission = 1.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS && hit.distance < surface.distance) transmission *= ring_transmission(S, ray, hit);
    }
    return transmission;
}

/* atmosphere: pathtrace.wgsl:1092-1213. Returns the in-scatter; the view
 * transmittance goes to *transmittance when given. */
static v3 atmosphere(const scene *S, v3 origin, v3 dir, real limit, uint32_t *rng, v3 *transmittance) {
    if (transmittance) *transmittance = V(1, 1, 1);
    if (S->s->g.atmo_params[3] < 0.5f) return V(0, 0, 0);
    real exit_ = shell_exit(S, origin, dir);
    real t_max = minf_(limit, exit_);
    if (t_max <= 0.0f) return V(0, 0, 0);
    v3 beta_ext = beta_extinction(S);
    real r = host_radius(S);
    uint32_t steps = view_steps(t_max / (0.25f * atmo_scale_height(S)));
    real dt = t_max / (real)steps;
    /* select() evaluates both operands: the draw is always taken. */
    uint32_t jitter_rng = hash_u32(*rng ^ 0x3c6ef372u);
    real jittered = rnd(S, &jitter_rng);
    real jitter = (steps < ATMO_VIEW_STEPS || limit < exit_) ? jittered : 0.5f;

    uint32_t reflected_rng = hash_u32(*rng ^ 0xa511e9b3u);
    reflector_t reflector = sample_reflector(S, origin, &reflected_rng);
    v3 reflected = V(0, 0, 0), reflected_direction = dir, reflected_phase = V(0, 0, 0);
    if (reflector.index != MISS) {
        ray_t reflected_ray = {origin, dir, MISS};
        light_sample light = sample_light(S, reflected_ray, reflector.index, &reflected_rng);
        reflected_ray.dir = light.dir;
        reflected = vmul(reflected_radiance(S, reflected_ray, reflector.index, &reflected_rng),
                         reflector.inverse_probability / light.pdf);
        reflected_direction = light.dir;
        reflected_phase = phase_weight(S, vdot(dir, light.dir));
    }
    if (reflected.x > 0.0f || reflected.y > 0.0f || reflected.z > 0.0f) {
        real sun = brightest_risen_light(S, origin);
        if (sun > 0.0f) {
            real ratio = maxf_(reflected.x, maxf_(reflected.y, reflected.z)) / sun;
            real minimum = 1.0f / r_sqrt(clampf_((real)S->s->counts[1] + 1.0f, 1.0f, 4096.0f));
            real keep = clampf_(ratio * 1.0e3f, minimum, 1.0f);
            reflected = rnd(S, &reflected_rng) < keep ? vdivs(reflected, keep) : V(0, 0, 0);
        }
    }
    int planetshine = reflected.x > 0.0f || reflected.y > 0.0f || reflected.z > 0.0f;

    v3 t_view = V(1, 1, 1), inscatter = V(0, 0, 0);
    for (uint32_t i = 0; i < steps; i++) {
        v3 p = vadd(origin, vmul(dir, ((real)i + jitter) * dt));
        v3 to_center = vsub(p, atmo_center(S));
        real altitude = maxf_(vlength(to_center) - r, 0.0f);
        real density = r_exp(-altitude / atmo_scale_height(S));
        real column = density * dt;
        v3 tau = vmul(beta_ext, column);
        v3 step_t = V(r_exp(-tau.x), r_exp(-tau.y), r_exp(-tau.z));
        v3 segment;
        segment.x = tau.x < 1.0e-3f ? column * (1.0f - 0.5f * tau.x) : (1.0f - step_t.x) / maxf_(beta_ext.x, 1.0e-20f);
        segment.y = tau.y < 1.0e-3f ? column * (1.0f - 0.5f * tau.y) : (1.0f - step_t.y) / maxf_(beta_ext.y, 1.0e-20f);
        segment.z = tau.z < 1.0e-3f ? column * (1.0f - 0.5f * tau.z) : (1.0f - step_t.z) / maxf_(beta_ext.z, 1.0e-20f);
        for (uint32_t slot = 0; slot < light_count(S); slot++) {
            uint32_t b = light_index(S, slot);
            if (b_emissive(S, b) < 0.5f) continue;
            ray_t light_ray = {p, dir, MISS};
            uint32_t light_samples = eclipse_light_samples(S, light_ray, b);
            for (uint32_t k = 0; k < light_samples; k++) {
                light_sample light = sample_light_stratum(S, light_ray, b, k, light_samples, rng);
                light_ray.dir = light.dir;
                real visibility = air_light_visibility(S, light_ray, b);
                if (visibility == 0.0f) continue;
                v3 e_sun = vmul(b_color(S, b), visibility / ((real)light_samples * light.pdf));
                v3 sun_t = vexp_neg(beta_ext, density_integral(S, p, light.dir, ATMO_SUN_STEPS));
                v3 beta_phase = phase_weight(S, vdot(dir, light.dir));
                inscatter = vadd(inscatter, vmulv(vmulv(vmulv(vmulv(t_view, segment), beta_phase), e_sun), sun_t));
            }
        }
        if (planetshine) {
            ray_t shine = {p, reflected_direction, MISS};
            real visibility = air_light_visibility(S, shine, reflector.index);
            if (visibility > 0.0f) {
                v3 light_t = vexp_neg(beta_ext, density_integral(S, p, reflected_direction, ATMO_SUN_STEPS));
                inscatter = vadd(inscatter, vmulv(vmulv(vmulv(vmulv(t_view, segment), reflected_phase), reflected),
                                                  vmul(light_t, visibility)));
            }
        }
        t_view = vmulv(t_view, step_t);
    }
    if (transmittance) *transmittance = t_view;
    return inscatter;
}

/* camera_air_transmittance: pathtrace.wgsl:1217-1234 */
static v3 camera_air_transmittance(const scene *S, v3 origin, v3 dir, real limit, uint32_t seed) {
    real exit_ = shell_exit(S, origin, dir);
    real t_max = minf_(limit, exit_);
    if (t_max <= 0.0f) return V(1, 1, 1);
    uint32_t steps = view_steps(t_max / (0.25f * atmo_scale_height(S)));
    real dt = t_max / (real)steps;
    uint32_t jitter_rng = hash_u32(seed ^ 0x3c6ef372u);
    real jittered = rnd(S, &jitter_rng);
    real jitter = (steps < ATMO_VIEW_STEPS || limit < exit_) ? jittered : 0.5f;
    v3 beta_ext = beta_extinction(S);
    v3 transmittance = V(1, 1, 1);
    for (uint32_t i = 0; i < steps; i++) {
        v3 p = vadd(origin, vmul(dir, ((real)i + jitter) * dt));
        real altitude = maxf_(vlength(vsub(p, atmo_center(S))) - host_radius(S), 0.0f);
        real column = r_exp(-altitude / atmo_scale_height(S)) * dt;
        transmittance = vmulv(transmittance, vexp_neg(beta_ext, column));
    }
    return transmittance;
}

/* cache_surface_sky: terrain.wgsl:286-302 (128 texels, 16 azimuths x 8
 * elevations; settings of the frame's first dispatch). */
static void cache_surface_sky(const scene *S, real *out) {
    for (uint32_t index = 0; index < SKY_TEXELS; index++) {
        uint32_t x = index % 16u, y = index / 16u;
        v3 light = V(0, 0, 0);
        if (S->s->g.atmo_params[3] > 0.5f && S->s->g.ground_counts[1] != 0u) {
            real mu = ((real)y + 0.5f) / 8.0f;
            real phi = TAU_F * ((real)x + 0.5f) / 16.0f;
            real r = r_sqrt(1.0f - mu * mu);
            v3 dir = from_ground(S, V(r * r_cos(phi), mu, r * r_sin(phi)));
            uint32_t rng = hash_u32(index ^ 0x91ce452du);
            light = atmosphere(S, V(0, 0, 0), dir, 1.0e30f, &rng, NULL);
        }
        out[4 * index] = light.x;
        out[4 * index + 1] = light.y;
        out[4 * index + 2] = light.z;
        out[4 * index + 3] = 0.0f;
    }
}

/* surface_sky_texel, surface_sky_lookup: terrain.wgsl:303-315 */
static v3 surface_sky_texel(const scene *S, int x, int y) {
    int yy = y < 0 ? 0 : (y > 7 ? 7 : y);
    const real *t = S->sky + 4 * ((uint32_t)yy * 16u + (uint32_t)((x + 16) % 16));
    return V(t[0], t[1], t[2]);
}
static v3 surface_sky_lookup(const scene *S, v3 dir) {
    if (!S->sky) return V(0, 0, 0);
    v3 p = to_ground(S, dir);
    if (p.y <= 0.0f) return V(0, 0, 0);
    real ux = r_fmod(r_atan2(p.z, p.x) / TAU_F + 1.0f, 1.0f) * 16.0f - 0.5f;
    real uy = p.y * 8.0f - 0.5f;
    int cx = (int)r_floor(ux), cy = (int)r_floor(uy);
    real fx = ux - r_floor(ux), fy = uy - r_floor(uy);
    v3 a = v3mix(surface_sky_texel(S, cx, cy), surface_sky_texel(S, cx + 1, cy), fx);
    v3 b = v3mix(surface_sky_texel(S, cx, cy + 1), surface_sky_texel(S, cx + 1, cy + 1), fx);
    return v3mix(a, b, fy);
}

/* sky_blocked, surface_sky: terrain.wgsl:317-339 */
static int sky_blocked(const scene *S, ray_t ray) {
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (S->s->g.ground_north[3] == (real)(i + 1u)) continue;
        if (sphere_hit(S, ray, i).index != MISS) return 1;
    }
    return landscape_query(S, ray, 1.0e30f, 1).index != MISS;
}
static v3 surface_sky(const scene *S, ray_t origin, v3 normal, uint32_t *rng) {
    real u = rnd(S, rng);
    real phi = TAU_F * rnd(S, rng);
    v3 dir = basis_direction(normal, r_sqrt(u) * r_cos(phi), r_sqrt(u) * r_sin(phi), r_sqrt(1.0f - u));
    v3 light = surface_sky_lookup(S, dir);
    if (maxf_(light.x, maxf_(light.y, light.z)) <= 0.0f) return V(0, 0, 0);
    ray_t ray = {origin.offset, dir, origin.anchor};
    if (sky_blocked(S, ray)) return V(0, 0, 0);
    real transmission = 1.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS) transmission *= ring_transmission(S, ray, hit);
    }
    return vmul(light, transmission);
}

/* ---------------------------------------------------------------- */
/* trace: pathtrace.wgsl:1347-1617                                   */
/* With a direction D (adjoint check), dout receives the tangent of  */
/* the returned radiance along D: every sampling decision, pdf, MIS   */
/* weight and Russian-roulette survival keeps its value, only the     */
/* material factors (ring tables and albedo, colours, albedo map)     */
/* carry tangents. The ring-indirect cap is differentiated exactly.   */
/* ---------------------------------------------------------------- */
/* out[0..3]: radiance and the backdrop's luminance; out[4..6]: the backdrop. */
static void trace(const scene *S, ray_t initial, uint32_t *rng, real out[7], const oracle_direction *D,
                  real dout[3]) {
    const sg_settings *st = S->s;
    ray_t ray = initial;
    v3 throughput = V(1, 1, 1);
    v3 radiance = V(0, 0, 0);
    v3 backdrop = V(0, 0, 0);
    real previous_pdf = 0.0f;
    ray_t previous_vertex = initial;
    uint32_t depth = 0, null_crossings = 0;
    int point_gained = 0;
    real ring_cap = 1.0e30f;
    v3 ring_base = V(0, 0, 0);
    uint32_t shine_body = MISS;
    /* Host air (pathtrace.wgsl:1361-1368): the previous vertex lies in the
     * air; the previous vertex was a sky-lit local surface. */
    int in_air = 0, sky_on_escape = 0, camera_segment = 1;
    /* tangents: detached (sampling held fixed) everywhere; after the first
     * ring scatter also the full tangent (pdfs and MIS weights attached)
     * of the throughput and of the radiance gathered since, and the score
     * (d log probability) of the decisions taken since. */
    v3 dthroughput = V(0, 0, 0), dradiance = V(0, 0, 0);
    real dring_cap = 0.0f;
    int captured = 0;
    v3 dthroughput_full = V(0, 0, 0), dindirect_full = V(0, 0, 0);
    real score = 0.0f, dlog_previous_pdf = 0.0f;
    for (;;) {
        EV(vertices);
        hit_t hit = closest_hit(S, ray);
        real disc_scale = 1.0f;
        if (depth == 0u && null_crossings == 0u && st->background[3] > 0.0f)
            hit = point_disc_hit(S, ray, hit, &disc_scale, rng);
        ring_hit_t ring = closest_ring(S, ray, hit.distance);
        /* pathtrace.wgsl:1387-1414: extinction of a continuation that left
         * the air for a celestial surface or a ring, and the camera ray's
         * air (its in-scatter from integrate_camera_air). */
        if (in_air) {
            in_air = 0;
            uint32_t host = (uint32_t)st->g.atmo_params[3] - 1u;
            if (ring.index != MISS || (hit.index < LOCAL_BASE && hit.index != host))
                throughput = vmulv(throughput, air_transmittance(S, ray, ray.dir));
        }
        if (camera_segment) {
            camera_segment = 0;
            real limit = 1.0e30f;
            if (hit.index != MISS) limit = hit.distance;
            if (ring.index != MISS) limit = minf_(limit, ring.distance);
            if (st->g.atmo_params[3] >= 0.5f) {
                v3 transmittance = camera_air_transmittance(S, ray.offset, ray.dir, limit, *rng);
                radiance = vadd(radiance, vmulv(throughput, V(S->air->radiance[0], S->air->radiance[1],
                                                              S->air->radiance[2])));
                throughput = vmulv(throughput, transmittance);
                *rng = S->air->rng;
            }
        }
        if (ring.index != MISS) {
            EV(ring_events);
            const sg_sphere *planet = &S->b[ring.index];
            if (depth == 0u && !point_gained && st->background[3] > 0.0f) {
                point_gained = 1;
                real gain = point_gain(S, planet->radius * planet->ring_params[0], ring.distance);
                throughput = vmul(throughput, gain);
                if (D) dthroughput = vmul(dthroughput, gain);
            }
            v3 n = b_pole(S, ring.index);
            optics_t optics = ring_optics(S, ring.index, ring.point);
            optics_t doptics = ring_optics_dot(S, D, ring.index, ring.point);
            real mu_out = vdot(vneg(ray.dir), n);
            real transmission = ring_transmission(S, ray, ring);
            real scatter_probability = one_minus_exp(optics.tau / maxf_(r_fabs(mu_out), 1.0e-7f));
            real bsdf_pdf = scatter_probability / (4.0f * PI_F);
            int last_vertex = depth + 1u == st->counts[3];
            /* d log scatter_probability and d log T along D */
            real dlog_pdf = 0.0f, dlog_t = 0.0f;
            if (D) {
                real m_out = maxf_(r_fabs(mu_out), 1.0e-7f);
                real x = optics.tau / m_out;
                if (scatter_probability > 0.0f)
                    dlog_pdf = (x < 1.0e-3f ? 1.0f - x : r_exp(-x)) * (doptics.tau / m_out) / scatter_probability;
                dlog_t = -doptics.tau / maxf_(r_fabs(vdot(ray.dir, n)), 1.0e-7f);
            }
            real ring_mis = 1.0f;
            if (shine_body == ring.index && null_crossings == 0u) {
                real cos_ring = maxf_(r_fabs(vdot(ray.dir, n)), 1.0e-6f);
                real shine_pdf = ring.distance * ring.distance / (ring_area(S, ring.index) * cos_ring);
                ring_mis = power_weight(previous_pdf, shine_pdf);
            }
            shine_body = MISS;
            real unshadowed = 0.0f, direct = 0.0f, dunshadowed = 0.0f, ddirect = 0.0f;
            uint32_t count = light_count(S);
            for (uint32_t slot = 0; slot < count; slot++) {
                uint32_t i = light_index(S, slot);
                if (b_emissive(S, i) < 0.5f || optics.tau == 0.0f) continue;
                ray_t origin = {ring.point, n, ring.index};
                light_sample light = sample_light(S, origin, i, rng);
                real mu_in = vdot(light.dir, n);
                ray_t shadow = ring_origin(S, ring, light.dir);
                real visibility = light_visibility(S, shadow, i);
                real weight = power_weight(light.pdf, bsdf_pdf);
                if (last_vertex) weight = 1.0f;
                v3 lit = vmul(vmulv(vmulv(throughput, ring_bsdf(optics, mu_out, mu_in)), b_color(S, i)),
                              r_fabs(mu_in) / light.pdf);
                radiance = vadd(radiance, vmul(lit, visibility * weight * ring_mis));
                unshadowed += lum(lit);
                direct += lum(lit) * visibility;
                if (D) {
                    v3 bsdf = ring_bsdf(optics, mu_out, mu_in);
                    v3 dbsdf = ring_bsdf_dot(optics, doptics, mu_out, mu_in);
                    v3 color = b_color(S, i), dcolor = dir_body_color(D, i);
                    v3 dlit = vmul(vadd(vadd(vmulv(vmulv(dthroughput, bsdf), color), vmulv(vmulv(throughput, dbsdf), color)),
                                        vmulv(vmulv(throughput, bsdf), dcolor)),
                                   r_fabs(mu_in) / light.pdf);
                    real dvis = light_visibility_dot(S, D, shadow, i, visibility);
                    dradiance = vadd(dradiance, vadd(vmul(dlit, visibility * weight * ring_mis),
                                                     vmul(lit, dvis * weight * ring_mis)));
                    dunshadowed += lum(dlit);
                    ddirect += lum(dlit) * visibility + lum(lit) * dvis;
                    if (captured) {
                        v3 dlit_full = vmul(vadd(vadd(vmulv(vmulv(dthroughput_full, bsdf), color),
                                                      vmulv(vmulv(throughput, dbsdf), color)),
                                                 vmulv(vmulv(throughput, bsdf), dcolor)),
                                            r_fabs(mu_in) / light.pdf);
                        real dweight = last_vertex ? 0.0f : weight * (-2.0f * (1.0f - weight)) * dlog_pdf;
                        dindirect_full = vadd(dindirect_full,
                                              vadd(vadd(vmul(dlit_full, visibility * weight * ring_mis),
                                                        vmul(lit, dvis * weight * ring_mis)),
                                                   vmul(lit, visibility * dweight * ring_mis)));
                    }
                }
            }
            if (rnd(S, rng) < transmission) {
                /* The crossing weighs exp(-tau / |mu|) at that probability:
                 * a detached factor; attached, the value is unchanged and
                 * the decision's score is d log T. */
                if (D) {
                    dthroughput = vadd(dthroughput, vmul(throughput, dlog_t));
                    score += dlog_t;
                }
                ray = ring_origin(S, ring, ray.dir);
                null_crossings += 1u;
                if (null_crossings > st->counts[0]) break;
                continue;
            }
            if (last_vertex || scatter_probability == 0.0f) break;
            if (ring_cap > 1.0e29f) {
                ring_cap = maxf_(direct, RING_INDIRECT_CAP * unshadowed);
                ring_base = radiance;
                dring_cap = direct >= RING_INDIRECT_CAP * unshadowed ? ddirect : RING_INDIRECT_CAP * dunshadowed;
                captured = 1;
                dthroughput_full = dthroughput;
                score = 0.0f;
            }
            real z = 1.0f - 2.0f * rnd(S, rng);
            real phi = TAU_F * rnd(S, rng);
            real radial = r_sqrt(maxf_(0.0f, 1.0f - z * z));
            v3 direction = basis_direction(n, radial * r_cos(phi), radial * r_sin(phi), z);
            if (D) {
                v3 bsdf = ring_bsdf(optics, mu_out, z);
                v3 dbsdf = ring_bsdf_dot(optics, doptics, mu_out, z);
                dthroughput = vmul(vadd(vmulv(dthroughput, bsdf), vmulv(throughput, dbsdf)), r_fabs(z) / bsdf_pdf);
                if (captured) {
                    v3 next = vmul(vmulv(throughput, bsdf), r_fabs(z) / bsdf_pdf);
                    dthroughput_full = vsub(vmul(vadd(vmulv(dthroughput_full, bsdf), vmulv(throughput, dbsdf)),
                                                 r_fabs(z) / bsdf_pdf),
                                            vmul(next, dlog_pdf));
                    score += transmission < 1.0f ? -dlog_t * transmission / (1.0f - transmission) : 0.0f;
                }
                dlog_previous_pdf = dlog_pdf;
            }
            throughput = vmul(vmulv(throughput, ring_bsdf(optics, mu_out, z)), r_fabs(z) / bsdf_pdf);
            previous_pdf = bsdf_pdf;
            sky_on_escape = 0;
            ray = ring_origin(S, ring, direction);
            previous_vertex = ray;
            depth += 1u;
            null_crossings = 0u;
            if (depth >= 3u) {
                real survival = clampf_(maxf_(throughput.x, maxf_(throughput.y, throughput.z)), 0.05f, 0.95f);
                int survived = rnd(S, rng) < survival;
                if (D && captured) roulette_tangent(throughput, survival, survived, &dthroughput_full, &score);
                if (!survived) break;
                throughput = vdivs(throughput, survival);
                if (D) dthroughput = vdivs(dthroughput, survival);
            }
            continue;
        }
        if (hit.index == MISS) {
            /* pathtrace.wgsl:1494-1508: background stars and the Milky Way
             * along unscattered camera paths (straight-through ring
             * crossings included); the backdrop is also returned apart. */
            if (sky_on_escape) radiance = vadd(radiance, vmulv(throughput, surface_sky_lookup(S, ray.dir)));
            if (depth == 0u) {
                radiance = vadd(radiance, vmulv(throughput, environment(S, ray.dir)));
                backdrop = vmulv(milky_way(S, ray.dir), throughput);
                radiance = vadd(radiance, backdrop);
            }
            break;
        }
        int local = hit.index >= LOCAL_BASE;
        uint32_t bi = hit.index;
        throughput = vmul(throughput, disc_scale);
        if (D) dthroughput = vmul(dthroughput, disc_scale);
        if (D && captured) dthroughput_full = vmul(dthroughput_full, disc_scale);
        if (!local && b_emissive(S, bi) > 0.5f) {
            real weight = 1.0f;
            if (depth > 0u) {
                real light_pdf = 1.0f / (TAU_F * cone_width(S, previous_vertex, hit.index));
                weight = power_weight(previous_pdf, light_pdf);
            }
            radiance = vadd(radiance, vmul(vmulv(throughput, b_color(S, bi)), weight));
            if (D)
                dradiance = vadd(dradiance, vmul(vadd(vmulv(dthroughput, b_color(S, bi)),
                                                      vmulv(throughput, dir_body_color(D, bi))), weight));
            if (D && captured) {
                real dweight = depth > 0u ? weight * 2.0f * (1.0f - weight) * dlog_previous_pdf : 0.0f;
                dindirect_full = vadd(dindirect_full,
                                      vadd(vmul(vadd(vmulv(dthroughput_full, b_color(S, bi)),
                                                     vmulv(throughput, dir_body_color(D, bi))), weight),
                                           vmul(vmulv(throughput, b_color(S, bi)), dweight)));
            }
            break;
        }
        EV(surface_events);
        if (!local && depth == 0u && !point_gained && st->background[3] > 0.0f) {
            point_gained = 1;
            real extent = S->b[bi].radius * maxf_(1.0f, S->b[bi].ring_params[0]);
            real gain = point_gain(S, extent, hit.distance);
            throughput = vmul(throughput, gain);
            if (D) dthroughput = vmul(dthroughput, gain);
            if (D && captured) dthroughput_full = vmul(dthroughput_full, gain);
        }
        v3 normal = local ? landscape_shading_normal(S, ray, hit) : hit.normal;
        ray_t outgoing;
        if (local) {
            outgoing = landscape_outgoing(S, ray, hit);
        } else {
            outgoing.offset = vmul(normal, S->b[bi].radius * (1.0f + 2.0e-6f));
            outgoing.dir = normal;
            outgoing.anchor = hit.index;
        }
        /* The guided ground sampler (src/guided_ground.rs:38-48). */
        reflector_t ground_reflector = {MISS, 0.0f};
        if (S->t && S->t->guided_ground && local && depth == 0u && st->g.atmo_params[3] > 0.5f)
            ground_reflector = sample_reflector(S, camera_origin(S, outgoing), rng);
        int guided = ground_reflector.index != MISS;
        v3 direct_light = V(0, 0, 0), ddirect_light = V(0, 0, 0);
        int last_vertex = depth + 1u == st->counts[3];
        uint32_t count = light_count(S);
        for (uint32_t slot = 0; slot < count; slot++) {
            uint32_t i = light_index(S, slot);
            if (b_emissive(S, i) < 0.5f) continue;
            light_sample sample = sample_light(S, outgoing, i, rng);
            real cosine = maxf_(vdot(normal, sample.dir), 0.0f);
            if (cosine <= 0.0f) continue;
            outgoing.dir = sample.dir;
            real visibility = light_visibility(S, outgoing, i);
            if (visibility > 0.0f) {
                real bsdf_pdf = cosine / PI_F;
                real path_pdf = bsdf_pdf;
                if (guided) path_pdf = 0.5f * (bsdf_pdf + ground_reflector_pdf(S, outgoing));
                real weight = power_weight(sample.pdf, path_pdf);
                if (last_vertex) weight = 1.0f;
                v3 color = b_color(S, i);
                if (air_on(S)) color = vmulv(color, air_transmittance(S, outgoing, sample.dir));
                direct_light = vadd(direct_light, vmul(color, bsdf_pdf * weight * visibility / sample.pdf));
                if (D) {
                    real dvis = light_visibility_dot(S, D, outgoing, i, visibility);
                    ddirect_light = vadd(ddirect_light,
                                         vadd(vmul(dir_body_color(D, i), bsdf_pdf * weight * visibility / sample.pdf),
                                              vmul(b_color(S, i), bsdf_pdf * weight * dvis / sample.pdf)));
                }
            }
        }
        v3 albedo = local ? landscape_albedo(S, ray, hit) : surface_albedo(S, bi, normal);
        v3 dalbedo = V(0, 0, 0);
        if (D) dalbedo = local ? landscape_albedo_dot(S, D, ray, hit) : surface_albedo_dot(S, D, bi, normal);
        radiance = vadd(radiance, vmulv(vmulv(throughput, albedo), direct_light));
        if (D)
            dradiance = vadd(dradiance, vadd(vmulv(vadd(vmulv(dthroughput, albedo), vmulv(throughput, dalbedo)), direct_light),
                                             vmulv(vmulv(throughput, albedo), ddirect_light)));
        if (D && captured)
            dindirect_full = vadd(dindirect_full,
                                  vadd(vmulv(vadd(vmulv(dthroughput_full, albedo), vmulv(throughput, dalbedo)), direct_light),
                                       vmulv(vmulv(throughput, albedo), ddirect_light)));
        shine_body = MISS;
        if (!local && !(S->t && S->t->ringshine_off)) {
            v3 dshine = V(0, 0, 0);
            v3 shine = ringshine(S, hit.index, outgoing.offset, normal, last_vertex, rng, D, D ? &dshine : NULL);
            radiance = vadd(radiance, vmulv(vmulv(throughput, albedo), shine));
            if (D)
                dradiance = vadd(dradiance, vadd(vmulv(vadd(vmulv(dthroughput, albedo), vmulv(throughput, dalbedo)), shine),
                                                 vmulv(vmulv(throughput, albedo), dshine)));
            if (D && captured)
                dindirect_full = vadd(dindirect_full,
                                      vadd(vmulv(vadd(vmulv(dthroughput_full, albedo), vmulv(throughput, dalbedo)), shine),
                                           vmulv(vmulv(throughput, albedo), dshine)));
            shine_body = hit.index;
        }
        /* Sky light of local surfaces (pathtrace.wgsl:1578-1584): an
         * explicit sample at the depth limit, else the continuation's
         * escape (sky_on_escape). */
        int sky_lit = local && st->g.ground_counts[1] != 0u && st->g.atmo_params[3] > 0.5f;
        if (sky_lit && last_vertex)
            radiance = vadd(radiance, vmulv(vmulv(throughput, albedo), surface_sky(S, outgoing, normal, rng)));
        if (last_vertex) break;
        real u = rnd(S, rng);
        real phi = TAU_F * rnd(S, rng);
        real cosine = r_sqrt(1.0f - u);
        outgoing.dir = basis_direction(normal, r_sqrt(u) * r_cos(phi), r_sqrt(u) * r_sin(phi), cosine);
        previous_pdf = cosine / PI_F;
        /* src/guided_ground.rs:59-76 */
        real path_weight = 1.0f;
        if (guided) {
            if (rnd(S, rng) < 0.5f) outgoing.dir = sample_light(S, outgoing, ground_reflector.index, rng).dir;
            real sampled_cosine = maxf_(vdot(normal, outgoing.dir), 0.0f);
            if (sampled_cosine == 0.0f) break;
            real brdf_pdf = sampled_cosine / PI_F;
            previous_pdf = 0.5f * (brdf_pdf + ground_reflector_pdf(S, outgoing));
            path_weight = brdf_pdf / previous_pdf;
        }
        if (D) dthroughput = vadd(vmulv(dthroughput, albedo), vmulv(throughput, dalbedo));
        if (D && captured) dthroughput_full = vadd(vmulv(dthroughput_full, albedo), vmulv(throughput, dalbedo));
        dlog_previous_pdf = 0.0f;
        throughput = vmulv(throughput, vmul(albedo, path_weight));
        if (depth >= 2u) {
            real survival = clampf_(maxf_(throughput.x, maxf_(throughput.y, throughput.z)), 0.05f, 0.95f);
            int survived = rnd(S, rng) < survival;
            if (D && captured) roulette_tangent(throughput, survival, survived, &dthroughput_full, &score);
            if (!survived) break;
            throughput = vdivs(throughput, survival);
            if (D) dthroughput = vdivs(dthroughput, survival);
        }
        ray = outgoing;
        previous_vertex = outgoing;
        in_air = inside_air(S, outgoing);
        sky_on_escape = sky_lit;
        depth += 1u;
        null_crossings = 0u;
    }
    v3 dfinal = dradiance;
    if (ring_cap < 1.0e29f) {
        v3 indirect = vsub(radiance, ring_base);
        real luminance = lum(indirect);
        if (luminance > ring_cap) {
            radiance = vadd(ring_base, vmul(indirect, ring_cap / luminance));
            /* The clamp makes the estimator nonlinear in the radiance
             * gathered after the cap vertex (I), so holding that part's
             * sampling fixed is no longer unbiased. Split the result into
             * base + I (linear: detached tangent) and the correction
             * C = I (cap / lum(I) - 1), whose tangent is the attached one
             * plus C times the score of the decisions from the cap vertex's
             * scatter on (likelihood ratio). */
            v3 hat = vdivs(indirect, luminance);
            v3 dq = vadd(vmul(hat, dring_cap),
                         vmul(vsub(dindirect_full, vmul(hat, lum(dindirect_full))), ring_cap / luminance));
            v3 correction = vmul(indirect, ring_cap / luminance - 1.0f);
            dfinal = vadd(vadd(dradiance, vsub(dq, dindirect_full)), vmul(correction, score));
        }
    }
    out[0] = radiance.x;
    out[1] = radiance.y;
    out[2] = radiance.z;
    out[3] = lum(backdrop);
    out[4] = backdrop.x;
    out[5] = backdrop.y;
    out[6] = backdrop.z;
    if (dout) {
        dout[0] = dfinal.x;
        dout[1] = dfinal.y;
        dout[2] = dfinal.z;
    }
}

/* camera_direction: pathtrace.wgsl:1619-1626 */
static v3 camera_direction(const scene *S, uint32_t x, uint32_t y, uint32_t *rng) {
    real jx = rnd(S, rng);
    real jy = rnd(S, rng);
    real u = ((real)x + jx) / S->s->g.viewport[0];
    real v = ((real)y + jy) / S->s->g.viewport[1];
    real ndc_x = 2.0f * u - 1.0f;
    real ndc_y = 1.0f - 2.0f * v;
    real tangent = S->s->g.cam_forward[3];
    return vnormalize(V(ndc_x * tangent * S->s->g.viewport[3], ndc_y * tangent, -1.0f));
}

/* Frames the restatement covers: landscape themes 0-5; terrain only with
 * a terrain table. */
static int check_frame_t(const sg_settings *s, const oracle_tables *t) {
    if (!s) return SG_ERR_INVALID;
    if (s->counts[0] > SG_BODY_CAPACITY) return SG_ERR_CAPACITY;
    if (s->g.ground_north[3] != 0.0f) {
        uint32_t theme = s->g.ground_counts[2] & 255u;
        if (theme > 5u) return SG_ERR_INVALID;
        if (s->g.ground_counts[1] != 0u && (!t || !t->terrain)) return SG_ERR_INVALID;
        if (s->g.ground_counts[0] > 0u && (!t || !t->ground || t->n_ground < s->g.ground_counts[0])) return SG_ERR_INVALID;
    }
    return SG_OK;
}
#define check_frame(s) check_frame_t((s), tables)

static void sample_pixel_d(const scene *S, uint32_t x, uint32_t y, uint32_t s, real out[7],
                           const oracle_direction *D, real dout[3]) {
    uint32_t width = (uint32_t)S->s->g.viewport[0];
    uint32_t pixel = y * width + x;
    uint32_t rng = hash_u32(pixel ^ hash_u32(S->s->sampling[0] + s + 0x9e3779b9u));
    ray_t ray;
    ray.offset = V(0, 0, 0);
    ray.dir = camera_direction(S, x, y, &rng);
    ray.anchor = MISS;
    trace(S, ray, &rng, out, D, dout);
}
static void sample_pixel(const scene *S, uint32_t x, uint32_t y, uint32_t s, real out[7]) {
    sample_pixel_d(S, x, y, s, out, NULL, NULL);
}

/* The surface sky cache as the frame's first dispatch builds it
 * (src/pathtracer.rs:946-954: only while the history holds no samples). */
static void prepare_sky(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                        real sky[4 * SKY_TEXELS]) {
    sg_settings first = *settings;
    first.counts[1] = 0u;
    scene S = {&first, bodies, tables, NULL, NULL, NULL};
    cache_surface_sky(&S, sky);
}

/* Sample `s` of a dispatch with host air: one integrate_camera_air / main
 * pair over a settings slice whose sampling.x and counts.y carry the
 * sample (src/pathtracer.rs:862-882, :963-968; pathtrace.wgsl:1629-1643). */
static void sample_pixel_air(const scene *S, uint32_t x, uint32_t y, uint32_t s, real out[7]) {
    sg_settings one = *S->s;
    one.sampling[0] = S->s->sampling[0] + s;
    one.counts[1] = S->s->counts[1] + s;
    one.counts[2] = 1u;
    scene A = *S;
    A.s = &one;
    uint32_t pixel = y * (uint32_t)one.g.viewport[0] + x;
    uint32_t rng = hash_u32(pixel ^ hash_u32(one.sampling[0] + 0x9e3779b9u));
    ray_t ray;
    ray.offset = V(0, 0, 0);
    ray.dir = camera_direction(&A, x, y, &rng);
    ray.anchor = MISS;
    hit_t hit = closest_hit(&A, ray);
    real disc_scale = 1.0f;
    if (one.background[3] > 0.0f) hit = point_disc_hit(&A, ray, hit, &disc_scale, &rng);
    ring_hit_t ring = closest_ring(&A, ray, hit.distance);
    v3 light = atmosphere(&A, ray.offset, ray.dir, minf_(hit.distance, ring.distance), &rng, NULL);
    camera_air_t air = {{light.x, light.y, light.z}, rng};
    A.air = &air;
    sample_pixel(&A, x, y, 0u, out);
}

/* main: pathtrace.wgsl:1645-1675 */
int oracle_dispatch(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                    float *accumulation, float *backdrop, uint32_t y0, uint32_t y1, int threads,
                    oracle_events *events) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    uint32_t width = (uint32_t)settings->g.viewport[0];
    uint32_t height = (uint32_t)settings->g.viewport[1];
    if (y1 > height) y1 = height;
    if (!accumulation || !backdrop || y0 > y1) return SG_ERR_INVALID;
    uint32_t z = settings->counts[2];
    if (z == 0u) return SG_OK;
    long total = (long)(y1 - y0) * (long)width;
#ifdef _OPENMP
    int nthreads = threads > 0 ? threads : omp_get_max_threads();
#else
    int nthreads = 1;
    (void)threads;
#endif
    oracle_events *per_thread = NULL;
    if (events) {
        per_thread = (oracle_events *)calloc((size_t)nthreads, sizeof(oracle_events));
        if (!per_thread) return SG_ERR_OOM;
    }
    const int air = settings->g.atmo_params[3] >= 0.5f;
    real sky[4 * SKY_TEXELS];
    if (air) prepare_sky(settings, bodies, tables, sky);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long k = 0; k < total; k++) {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        scene S = {settings, bodies, tables, per_thread ? &per_thread[tid] : NULL, air ? sky : NULL, NULL};
        uint32_t x = (uint32_t)(k % width);
        uint32_t y = y0 + (uint32_t)(k / width);
        uint32_t pixel = y * width + x;
        if (air) {
            /* One running-mean fold per sample, as the per-sample
             * dispatches of an air frame do. */
            for (uint32_t s = 0; s < z; s++) {
                real r[7];
                if (S.ev) S.ev->samples++;
                sample_pixel_air(&S, x, y, s, r);
                uint32_t old_count = settings->counts[1] + s;
                real w = 1.0f / (real)(old_count + 1u);
                for (int c = 0; c < 4; c++) {
                    real old = accumulation[4 * pixel + c];
                    accumulation[4 * pixel + c] = old_count > 0u ? old + (r[c] - old) * w : r[c];
                }
                for (int c = 0; c < 3; c++) {
                    real old = backdrop[4 * pixel + c];
                    backdrop[4 * pixel + c] = old_count > 0u ? old + (r[4 + c] - old) * w : r[4 + c];
                }
                backdrop[4 * pixel + 3] = 0.0f;
            }
            continue;
        }
        real sum[4] = {0, 0, 0, 0}, bsum[3] = {0, 0, 0};
        for (uint32_t s = 0; s < z; s++) {
            real r[7];
            if (S.ev) S.ev->samples++;
            sample_pixel(&S, x, y, s, r);
            for (int c = 0; c < 4; c++) sum[c] += r[c];
            for (int c = 0; c < 3; c++) bsum[c] += r[4 + c];
        }
        uint32_t old_count = settings->counts[1];
        uint32_t new_count = old_count + z;
        real mean[4], bmean[3];
        for (int c = 0; c < 4; c++) mean[c] = sum[c] / (real)z;
        for (int c = 0; c < 3; c++) bmean[c] = bsum[c] / (real)z;
        if (old_count > 0u) {
            real w = (real)z / (real)new_count;
            for (int c = 0; c < 4; c++) {
                real old = accumulation[4 * pixel + c];
                mean[c] = old + (mean[c] - old) * w;
            }
            for (int c = 0; c < 3; c++) {
                real old = backdrop[4 * pixel + c];
                bmean[c] = old + (bmean[c] - old) * w;
            }
        }
        for (int c = 0; c < 4; c++) accumulation[4 * pixel + c] = mean[c];
        for (int c = 0; c < 3; c++) backdrop[4 * pixel + c] = bmean[c];
        backdrop[4 * pixel + 3] = 0.0f;
    }
    if (events) {
        for (int t = 0; t < nthreads; t++) {
            uint64_t *dst = (uint64_t *)events;
            const uint64_t *src = (const uint64_t *)&per_thread[t];
            for (size_t f = 0; f < sizeof(oracle_events) / sizeof(uint64_t); f++) dst[f] += src[f];
        }
        free(per_thread);
    }
    return SG_OK;
}

int oracle_tangent(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                   const oracle_direction *direction, float *primal, float *tangent, uint32_t y0, uint32_t y1,
                   int threads) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    /* The adjoint does not differentiate the host air or the procedural
     * surface styles. */
    if (settings->g.atmo_params[3] >= 0.5f) return SG_ERR_INVALID;
    for (uint32_t i = 0; i < settings->counts[0]; i++)
        if (bodies[i].axis_x[3] >= 0.5f) return SG_ERR_INVALID;
    uint32_t width = (uint32_t)settings->g.viewport[0];
    uint32_t height = (uint32_t)settings->g.viewport[1];
    if (y1 > height) y1 = height;
    if (!primal || !tangent || !direction || y0 > y1) return SG_ERR_INVALID;
    uint32_t z = settings->counts[2];
    long total = (long)(y1 - y0) * (long)width;
#ifdef _OPENMP
    int nthreads = threads > 0 ? threads : omp_get_max_threads();
#else
    int nthreads = 1;
    (void)threads;
#endif
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long k = 0; k < total; k++) {
        scene S = {settings, bodies, tables, NULL, NULL, NULL};
        uint32_t x = (uint32_t)(k % width);
        uint32_t y = y0 + (uint32_t)(k / width);
        size_t pixel = (size_t)y * width + x;
        for (uint32_t s = 0; s < z; s++) {
            real r[7], d[3];
            sample_pixel_d(&S, x, y, s, r, direction, d);
            for (int c = 0; c < 4; c++) primal[4 * pixel + c] += r[c];
            for (int c = 0; c < 3; c++) tangent[4 * pixel + c] += d[c];
        }
    }
    return SG_OK;
}

int oracle_trace_sample(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                        uint32_t x, uint32_t y, uint32_t s, float out[4]) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL, NULL, NULL};
    real r[7];
    if (settings->g.atmo_params[3] >= 0.5f) {
        real sky[4 * SKY_TEXELS];
        prepare_sky(settings, bodies, tables, sky);
        S.sky = sky;
        sample_pixel_air(&S, x, y, s, r);
    } else {
        sample_pixel(&S, x, y, s, r);
    }
    for (int c = 0; c < 4; c++) out[c] = r[c];
    return SG_OK;
}

static ray_t to_ray(const sg_ray *r) {
    ray_t ray;
    ray.offset = V(r->offset[0], r->offset[1], r->offset[2]);
    ray.dir = V(r->direction[0], r->direction[1], r->direction[2]);
    ray.anchor = r->anchor;
    return ray;
}

int oracle_closest_hit(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                       const sg_ray *rays, uint32_t n, sg_hit *hits) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL, NULL, NULL};
    for (uint32_t i = 0; i < n; i++) {
        hit_t h = closest_hit(&S, to_ray(&rays[i]));
        hits[i].distance = h.distance;
        hits[i].index = h.index;
        hits[i].normal[0] = h.normal.x;
        hits[i].normal[1] = h.normal.y;
        hits[i].normal[2] = h.normal.z;
    }
    return SG_OK;
}

int oracle_light_visibility(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                            const sg_ray *rays, const uint32_t *lights, uint32_t n, float *out) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL, NULL, NULL};
    for (uint32_t i = 0; i < n; i++) out[i] = light_visibility(&S, to_ray(&rays[i]), lights[i]);
    return SG_OK;
}

int oracle_reference_visibility(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                                const sg_ray *rays, const uint32_t *lights, uint32_t n, float *out) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL, NULL, NULL};
    for (uint32_t k = 0; k < n; k++) {
        ray_t ray = to_ray(&rays[k]);
        hit_t surface = closest_hit(&S, ray);
        if (surface.index != lights[k]) { out[k] = 0.0f; continue; }
        real transmission = 1.0f;
        for (uint32_t i = 0; i < settings->counts[0]; i++) {
            ring_hit_t hit = ring_hit(&S, ray, i);
            if (hit.index != MISS && hit.distance < surface.distance) transmission *= ring_transmission(&S, ray, hit);
        }
        out[k] = transmission;
    }
    return SG_OK;
}

int oracle_ring_probe(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                      const sg_ray *rays, uint32_t body, uint32_t n, float *out) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    if (body >= settings->counts[0]) return SG_ERR_INVALID;
    scene S = {settings, bodies, tables, NULL, NULL, NULL};
    for (uint32_t i = 0; i < n; i++) {
        ray_t ray = to_ray(&rays[i]);
        ring_hit_t hit = ring_hit(&S, ray, body);
        if (hit.index == MISS) {
            out[4 * i] = out[4 * i + 1] = out[4 * i + 2] = out[4 * i + 3] = 0.0f;
            continue;
        }
        out[4 * i] = hit.distance;
        out[4 * i + 1] = vlength(hit.point) / bodies[body].radius;
        out[4 * i + 2] = ring_transmission(&S, ray, hit);
        out[4 * i + 3] = 1.0f;
    }
    return SG_OK;
}

float oracle_ring_energy(float albedo, float tau, float mu, uint32_t steps) {
    optics_t optics = {V(albedo, albedo, albedo), tau};
    real energy = r_exp(-optics.tau / mu);
    for (uint32_t i = 0; i < steps; i++) {
        real mi = ((real)i + 0.5f) / (real)steps;
        v3 sum = vadd(ring_bsdf(optics, mu, mi), ring_bsdf(optics, mu, -mi));
        energy += sum.x * (TAU_F * mi / (real)steps);
    }
    return energy;
}

int oracle_sample_light(const sg_settings *settings, const sg_sphere *bodies, const sg_ray *ray,
                        uint32_t light, uint32_t *rng, float direction[3], float *pdf) {
    scene S = {settings, bodies, NULL, NULL, NULL, NULL};
    light_sample ls = sample_light(&S, to_ray(ray), light, rng);
    direction[0] = ls.dir.x;
    direction[1] = ls.dir.y;
    direction[2] = ls.dir.z;
    *pdf = ls.pdf;
    return SG_OK;
}

int oracle_sky_cache(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                     float out[4 * 128]) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    real sky[4 * 128];
    prepare_sky(settings, bodies, tables, sky);
    for (int k = 0; k < 4 * 128; k++) out[k] = (float)sky[k];
    return SG_OK;
}

uint32_t oracle_hash(uint32_t value) { return hash_u32(value); }
float oracle_random(uint32_t *state) {
    scene S = {NULL, NULL, NULL, NULL, NULL, NULL};
    return rnd(&S, state);
}
