/*
 * oracle.c — CPU restatement of stargaze's progressive path-tracing
 * integrator. TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels,
 * never part of the product path. See oracle.h for the parity pin.
 *
 * Every function names the WGSL it restates. Expression order follows the
 * WGSL source; the file must be compiled with -ffp-contract=off and without
 * -ffast-math so that f32 + - * / sqrt round exactly as written.
 *
 * Scope: the airless integrator of pathtrace.wgsl (sample loop, spheres,
 * rings, stellar NEE with MIS, ringshine, point discs, Russian roulette,
 * running-mean accumulation) and rings.wgsl. The host atmosphere, catalogue
 * stars, Milky Way map, procedural surface styles 1-6 and the local
 * landscape are not restated: they are inert for the frames this oracle
 * accepts (atmo_params.w == 0, ground_north.w == 0).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
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
typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 vmul(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vmulv(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlength(v3 a) { return sqrtf(vdot(a, a)); }
static inline v3 vnormalize(v3 a) { float inv = 1.0f / sqrtf(vdot(a, a)); return vmul(a, inv); }
static inline float minf_(float a, float b) { return a < b ? a : b; }
static inline float maxf_(float a, float b) { return a > b ? a : b; }
static inline float clampf_(float x, float lo, float hi) { return minf_(maxf_(x, lo), hi); }
static inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
static inline float fractf(float x) { return x - floorf(x); }
static inline float smoothstepf(float e0, float e1, float x) {
    float t = clampf_((x - e0) / (e1 - e0), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
static inline float lum(v3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

/* ---------------------------------------------------------------- */
/* Scene access                                                      */
/* ---------------------------------------------------------------- */
typedef struct {
    const sg_settings *s;
    const sg_sphere *b;
    const oracle_tables *t;
    oracle_events *ev;
} scene;

typedef struct { v3 offset; v3 dir; uint32_t anchor; } ray_t;   /* pathtrace.wgsl:70-76 */
typedef struct { float distance; uint32_t index; v3 normal; } hit_t; /* :77-81 */
typedef struct { v3 dir; float pdf; } light_sample; /* :82-85 */
typedef struct { float distance; uint32_t index; v3 point; } ring_hit_t; /* rings.wgsl:2-6 */

static inline v3 b_center(const scene *S, uint32_t i) { return V(S->b[i].center[0], S->b[i].center[1], S->b[i].center[2]); }
static inline v3 b_low(const scene *S, uint32_t i) { return V(S->b[i].center_low[0], S->b[i].center_low[1], S->b[i].center_low[2]); }
static inline float b_radius(const scene *S, uint32_t i) { return S->b[i].radius; }
static inline v3 b_color(const scene *S, uint32_t i) { return V(S->b[i].color[0], S->b[i].color[1], S->b[i].color[2]); }
static inline float b_emissive(const scene *S, uint32_t i) { return S->b[i].emissive; }
static inline v3 b_pole(const scene *S, uint32_t i) { return V(S->b[i].ring_plane[0], S->b[i].ring_plane[1], S->b[i].ring_plane[2]); }
#define EV(field) do { if (S->ev) S->ev->field++; } while (0)

/* hash, random: pathtrace.wgsl:87-98 */
static inline uint32_t hash_u32(uint32_t value) {
    uint32_t x = value;
    x = (x ^ (x >> 16)) * 0x7feb352du;
    x = (x ^ (x >> 15)) * 0x846ca68bu;
    return x ^ (x >> 16);
}
static inline float rnd(const scene *S, uint32_t *state) {
    EV(rng_draws);
    *state = *state * 747796405u + 2891336453u;
    uint32_t word = ((*state >> ((*state >> 28) + 4u)) ^ *state) * 277803737u;
    return (float)(((word >> 22) ^ word) >> 8) * (1.0f / 16777216.0f);
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
static hit_t sphere_hit_radius(const scene *S, ray_t ray, uint32_t index, float radius) {
    EV(sphere_tests);
    v3 oc = relative_center(S, ray, index);
    float a = vdot(ray.dir, ray.dir);
    float b = vdot(oc, ray.dir);
    v3 pc = vcross(oc, ray.dir);
    float h = a * radius * radius - vdot(pc, pc);
    if (h < 0.0f) return miss_hit();
    float root = sqrtf(h);
    float q = b + (b >= 0.0f ? root : -root);
    if (q == 0.0f) return miss_hit();
    float c = vdot(oc, oc) - radius * radius;
    float near_ = (b < 0.0f) ? q / a : c / q;
    float far_ = (b < 0.0f) ? c / q : q / a;
    float distance = near_;
    float delta = -root / a;
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

/* landscape_query: ground.wgsl:123-242. The oracle accepts only frames
 * with the landscape disabled (ground_north.w == 0), where it returns the
 * initial closest record (ground.wgsl:124-125). */
static hit_t landscape_query(const scene *S, ray_t ray, float limit, int occlusion) {
    (void)ray; (void)occlusion; (void)S;
    hit_t h = {limit, MISS, {0, 0, 0}};
    return h;
}

/* closest_hit: pathtrace.wgsl:173-185 */
static hit_t closest_hit(const scene *S, ray_t ray) {
    hit_t closest = miss_hit();
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (S->s->g.ground_north[3] == (float)(i + 1u)) continue;
        hit_t hit = sphere_hit(S, ray, i);
        if (hit.distance < closest.distance) closest = hit;
    }
    hit_t local = landscape_query(S, ray, 1.0e30f, 0);
    if (local.distance < closest.distance) closest = local;
    return closest;
}

/* basis_direction: pathtrace.wgsl:187-194 */
static v3 basis_direction(v3 axis, float x, float y, float z) {
    v3 helper = V(0.0f, 0.0f, 1.0f);
    if (fabsf(axis.z) > 0.9f) helper = V(0.0f, 1.0f, 0.0f);
    v3 tangent = vnormalize(vcross(helper, axis));
    return vnormalize(vadd(vadd(vmul(tangent, x), vmul(vcross(axis, tangent), y)), vmul(axis, z)));
}

/* cone_width: pathtrace.wgsl:197-202 */
static float cone_width(const scene *S, ray_t ray, uint32_t index) {
    v3 oc = relative_center(S, ray, index);
    float r = b_radius(S, index);
    float sin2 = clampf_(r * r / vdot(oc, oc), 1.0e-20f, 1.0f);
    return sin2 / (1.0f + sqrtf(1.0f - sin2));
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
    float width = cone_width(S, ray, index);
    float radial = rnd(S, rng);
    float azimuth = rnd(S, rng);
    if (count == 4u) {
        radial = ((float)(stratum & 1u) + radial) * 0.5f;
        azimuth = ((float)(stratum >> 1u) + azimuth) * 0.5f;
    }
    float one_minus_cos = radial * width;
    float sin_theta = sqrtf(one_minus_cos * (2.0f - one_minus_cos));
    float phi = TAU_F * azimuth;
    light_sample ls;
    ls.dir = basis_direction(axis, sin_theta * cosf(phi), sin_theta * sinf(phi), 1.0f - one_minus_cos);
    ls.pdf = 1.0f / (TAU_F * width);
    return ls;
}
static inline light_sample sample_light(const scene *S, ray_t ray, uint32_t index, uint32_t *rng) {
    return sample_light_stratum(S, ray, index, 0u, 1u, rng);
}

/* power_weight: pathtrace.wgsl:264-267 */
static inline float power_weight(float a, float b) {
    float ratio = b / maxf_(a, 1.0e-30f);
    return 1.0f / (1.0f + ratio * ratio);
}

/* ---------------------------------------------------------------- */
/* Rings: rings.wgsl                                                 */
/* ---------------------------------------------------------------- */
static inline ring_hit_t ring_miss(float limit) { ring_hit_t r = {limit, MISS, {0, 0, 0}}; return r; }

/* ring_hit: rings.wgsl:8-34 */
static ring_hit_t ring_hit(const scene *S, ray_t ray, uint32_t index) {
    const sg_sphere *body = &S->b[index];
    if (body->ring_params[0] <= body->ring_plane[3] || body->ring_params[1] <= 0.0f) return ring_miss(1.0e30f);
    EV(ring_tests);
    v3 n = b_pole(S, index);
    float denom = vdot(ray.dir, n);
    if (fabsf(denom) < 1.0e-7f) return ring_miss(1.0e30f);
    v3 oc = relative_center(S, ray, index);
    float a = vdot(ray.dir, ray.dir);
    v3 perpendicular = vdivs(vcross(ray.dir, vcross(ray.dir, oc)), a);
    float along = -vdot(perpendicular, n) / denom;
    float distance = vdot(oc, ray.dir) / a + along;
    if (distance <= 0.0f) return ring_miss(1.0e30f);
    v3 point = vadd(perpendicular, vmul(ray.dir, along));
    float radius = vlength(point) / body->radius;
    if (radius < body->ring_plane[3] || radius > body->ring_params[0]) return ring_miss(1.0e30f);
    ring_hit_t r = {distance, index, point};
    return r;
}

/* closest_ring: rings.wgsl:36-45 */
static ring_hit_t closest_ring(const scene *S, ray_t ray, float limit) {
    ring_hit_t closest = ring_miss(limit);
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS && hit.distance < closest.distance) closest = hit;
    }
    return closest;
}

typedef struct { v3 color; float tau; } optics_t;

/* ring_optics: rings.wgsl:50-81, plus the tabulated-profile extension
 * (ring_params.w = slot + 1): tau = ring_params.y * table[bin(x)]. */
static optics_t ring_optics(const scene *S, uint32_t index, v3 point) {
    const sg_sphere *body = &S->b[index];
    float radius = vlength(point) / body->radius;
    float x = (radius - body->ring_plane[3]) / (body->ring_params[0] - body->ring_plane[3]);
    float tau = body->ring_params[1];
    v3 color = V(body->ring_color[0], body->ring_color[1], body->ring_color[2]);
    if (body->ring_params[3] >= 0.5f) {
        uint32_t slot = (uint32_t)body->ring_params[3] - 1u;
        const float *table = (S->t && slot < SG_RING_TABLE_SLOTS) ? S->t->ring_tau[slot] : NULL;
        uint32_t bins = table ? S->t->ring_bins[slot] : 0u;
        if (bins > 0u) {
            float fb = x * (float)bins;
            uint32_t bin = fb <= 0.0f ? 0u : (uint32_t)fb;
            if (bin > bins - 1u) bin = bins - 1u;
            tau *= table[bin];
        } else {
            tau = 0.0f;
        }
    } else if (body->ring_params[2] > 0.5f) {
        float broad = 0.5f + 0.5f * sinf(43.0f * x + 1.8f * sinf(17.0f * x));
        float fine = 0.5f + 0.5f * sinf(1900.0f * x + 2.0f * sinf(311.0f * x));
        float micro = 0.5f + 0.5f * sinf(6100.0f * x);
        float density = 0.12f;
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
        if (fabsf(x - 0.9487f) < 0.00262f || fabsf(x - 0.99565f) < 0.00034f) density = 0.0f;
        tau *= density;
        color = vmul(vmulv(color, tint), 0.94f + 0.06f * broad);
    }
    optics_t o = {color, tau};
    return o;
}

/* ring_transmission: rings.wgsl:83-86 */
static float ring_transmission(const scene *S, ray_t ray, ring_hit_t hit) {
    float mu = maxf_(fabsf(vdot(ray.dir, b_pole(S, hit.index))), 1.0e-7f);
    return expf(-ring_optics(S, hit.index, hit.point).tau / mu);
}

/* light_visibility: rings.wgsl:90-115 */
static float light_visibility(const scene *S, ray_t ray, uint32_t light) {
    EV(shadow_rays);
    hit_t surface = sphere_hit(S, ray, light);
    if (surface.index == MISS) return 0.0f;
    if (S->s->g.ground_north[3] == (float)(light + 1u) && closest_hit(S, ray).index != light) return 0.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (i == light || S->s->g.ground_north[3] == (float)(i + 1u)) continue;
        hit_t hit = sphere_hit(S, ray, i);
        if (hit.index != MISS && (hit.distance < surface.distance ||
                                  (hit.distance == surface.distance && i < light)))
            return 0.0f;
    }
    hit_t local = landscape_query(S, ray, surface.distance, 1);
    if (local.index != MISS && local.distance < surface.distance) return 0.0f;
    float transmission = 1.0f;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        ring_hit_t hit = ring_hit(S, ray, i);
        if (hit.index != MISS && hit.distance < surface.distance) transmission *= ring_transmission(S, ray, hit);
    }
    return transmission;
}

/* one_minus_exp: rings.wgsl:143-145 */
static inline float one_minus_exp(float x) {
    return x < 1.0e-3f ? x * (1.0f - 0.5f * x) : 1.0f - expf(-x);
}

/* ring_bsdf: rings.wgsl:151-166 */
static v3 ring_bsdf(optics_t optics, float outgoing, float incoming) {
    float mo = maxf_(fabsf(outgoing), 1.0e-7f);
    float mi = maxf_(fabsf(incoming), 1.0e-7f);
    float a = optics.tau / mo;
    float b = optics.tau / mi;
    if (outgoing * incoming < 0.0f) {
        float delta = fabsf(a - b);
        float integral = delta < 1.0e-3f ? 1.0f - 0.5f * delta
                                         : one_minus_exp(delta) / maxf_(delta, 1.0e-20f);
        float factor = optics.tau / (mo * mi) * expf(-minf_(a, b)) * integral;
        return vmul(optics.color, factor / (4.0f * PI_F));
    }
    float factor = one_minus_exp(a + b) / (mo + mi);
    return vmul(optics.color, factor / (4.0f * PI_F));
}

/* ring_origin: rings.wgsl:168-175 */
static ray_t ring_origin(const scene *S, ring_hit_t hit, v3 direction) {
    v3 n = b_pole(S, hit.index);
    float sign = vdot(direction, n) >= 0.0f ? 1.0f : -1.0f;
    v3 point = vsub(hit.point, vmul(n, vdot(hit.point, n)));
    ray_t r;
    r.offset = vadd(point, vmul(n, sign * b_radius(S, hit.index) * 2.0e-6f));
    r.dir = direction;
    r.anchor = hit.index;
    return r;
}

/* ring_area: pathtrace.wgsl:1237-1241 */
static float ring_area(const scene *S, uint32_t index) {
    const sg_sphere *body = &S->b[index];
    float r = body->radius;
    return PI_F * r * r * (body->ring_params[0] * body->ring_params[0] - body->ring_plane[3] * body->ring_plane[3]);
}

/* ringshine: pathtrace.wgsl:1248-1296 */
static v3 ringshine(const scene *S, uint32_t index, v3 origin, v3 normal, int last_vertex, uint32_t *rng) {
    const sg_sphere *body = &S->b[index];
    if (body->ring_params[0] <= body->ring_plane[3] || body->ring_params[1] <= 0.0f) return V(0, 0, 0);
    v3 n = b_pole(S, index);
    float inner = body->ring_plane[3] * body->ring_plane[3];
    float outer = body->ring_params[0] * body->ring_params[0];
    float radius = sqrtf(mixf(inner, outer, rnd(S, rng))) * body->radius;
    float phi = TAU_F * rnd(S, rng);
    v3 point = vmul(basis_direction(n, cosf(phi), sinf(phi), 0.0f), radius);
    v3 offset = vsub(point, origin);
    float distance2 = vdot(offset, offset);
    float distance = sqrtf(distance2);
    v3 direction = vdivs(offset, distance);
    float cos_surface = vdot(normal, direction);
    float cos_ring = fabsf(vdot(direction, n));
    if (cos_surface <= 0.0f || cos_ring < 1.0e-6f) return V(0, 0, 0);
    ray_t blocker_ray = {origin, direction, index};
    hit_t blocker = sphere_hit(S, blocker_ray, index);
    if (blocker.index != MISS && blocker.distance < distance) return V(0, 0, 0);
    optics_t optics = ring_optics(S, index, point);
    if (optics.tau == 0.0f) return V(0, 0, 0);
    float mu_out = vdot(vneg(direction), n);
    v3 shine = V(0, 0, 0);
    uint32_t count = light_count(S);
    for (uint32_t slot = 0; slot < count; slot++) {
        uint32_t i = light_index(S, slot);
        if (b_emissive(S, i) < 0.5f) continue;
        ray_t from_ring = {point, n, index};
        light_sample light = sample_light(S, from_ring, i, rng);
        float mu_in = vdot(light.dir, n);
        ring_hit_t rh = {0.0f, index, point};
        float visibility = light_visibility(S, ring_origin(S, rh, light.dir), i);
        shine = vadd(shine, vmul(vmulv(ring_bsdf(optics, mu_out, mu_in), b_color(S, i)),
                                 fabsf(mu_in) * visibility / light.pdf));
    }
    float pdf = distance2 / (ring_area(S, index) * cos_ring);
    float weight = power_weight(pdf, cos_surface / PI_F);
    if (last_vertex) weight = 1.0f;
    return vmul(shine, cos_surface * weight / (PI_F * pdf));
}

/* point_disc_hit: pathtrace.wgsl:1308-1333 */
static hit_t point_disc_hit(const scene *S, ray_t ray, hit_t closest, float *scale, uint32_t *rng) {
    hit_t result = closest;
    float total = 0.0f;
    float pixel = 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
    float angle = clampf_(POINT_DISC_RADIUS, 0.7f * pixel, STAR_DOT_PIXELS * pixel);
    uint32_t host = (uint32_t)S->s->g.atmo_params[3] - 1u;
    for (uint32_t i = 0; i < S->s->counts[0]; i++) {
        if (i == host || S->s->g.ground_north[3] == (float)(i + 1u)) continue;
        float radius = b_radius(S, i);
        float drawn = angle * vlength(relative_center(S, ray, i));
        if (radius <= 0.0f || drawn <= radius) continue;
        hit_t hit = sphere_hit_radius(S, ray, i, drawn);
        if (hit.distance < closest.distance) {
            float ratio = (radius / drawn) * (radius / drawn);
            total += ratio;
            if (rnd(S, rng) * total < ratio) result = hit;
        }
    }
    if (total > 0.0f) *scale = total;
    return result;
}

/* point_gain: pathtrace.wgsl:1341-1345 */
static float point_gain(const scene *S, float extent, float distance) {
    float pixel = 2.0f * S->s->g.cam_forward[3] / maxf_(S->s->g.viewport[1], 1.0f);
    float pixels = 2.0f * extent / maxf_(distance, 1.0e-30f) / pixel;
    return mixf(S->s->background[3], 1.0f, smoothstepf(1.0f, 3.0f, pixels));
}

/* ---------------------------------------------------------------- */
/* Surface albedo, style 0 (pathtrace.wgsl:338-389, :897-925)        */
/* ---------------------------------------------------------------- */
static float hash31(v3 p) {
    v3 q = V(fractf(p.x * 0.1031f), fractf(p.y * 0.1030f), fractf(p.z * 0.0973f));
    float d = vdot(q, V(q.y + 33.33f, q.x + 33.33f, q.z + 33.33f));
    q = V(q.x + d, q.y + d, q.z + d);
    return fractf((q.x + q.y) * q.z);
}
static float vnoise(v3 p) {
    v3 i = V(floorf(p.x), floorf(p.y), floorf(p.z));
    v3 f = vsub(p, i);
    v3 u = V(f.x * f.x * (3.0f - 2.0f * f.x), f.y * f.y * (3.0f - 2.0f * f.y), f.z * f.z * (3.0f - 2.0f * f.z));
    float a = mixf(hash31(i), hash31(vadd(i, V(1, 0, 0))), u.x);
    float b = mixf(hash31(vadd(i, V(0, 1, 0))), hash31(vadd(i, V(1, 1, 0))), u.x);
    float c = mixf(hash31(vadd(i, V(0, 0, 1))), hash31(vadd(i, V(1, 0, 1))), u.x);
    float d = mixf(hash31(vadd(i, V(0, 1, 1))), hash31(vadd(i, V(1, 1, 1))), u.x);
    return mixf(mixf(a, b, u.y), mixf(c, d, u.y), u.z);
}
static v3 surface_albedo(const scene *S, uint32_t index, v3 normal) {
    const sg_sphere *body = &S->b[index];
    v3 x = V(body->axis_x[0], body->axis_x[1], body->axis_x[2]);
    v3 y = V(body->axis_y[0], body->axis_y[1], body->axis_y[2]);
    v3 local = V(vdot(normal, x), vdot(normal, y), vdot(normal, vcross(x, y)));
    float mottle = 1.0f;
    if (body->center_low[3] > 0.0f) {
        float seed = body->axis_y[3];
        v3 off = vmul(V(hash31(V(seed, 1.0f, 7.0f)), hash31(V(3.0f, seed, 5.0f)), hash31(V(9.0f, 2.0f, seed))), 512.0f);
        v3 p = vadd(vmul(local, 2.4f), off);
        float amplitude = 0.5f, noise = 0.0f;
        for (int octave = 0; octave < 5; octave++) {
            noise += amplitude * vnoise(p);
            p = vmul(p, 2.07f);
            amplitude *= 0.5f;
        }
        mottle = mixf(1.0f, 0.68f + 0.64f * noise, body->center_low[3]);
    }
    v3 c = vmul(b_color(S, index), mottle);
    return V(clampf_(c.x, 0, 1), clampf_(c.y, 0, 1), clampf_(c.z, 0, 1));
}

/* ---------------------------------------------------------------- */
/* trace: pathtrace.wgsl:1347-1617 (airless, landscape off)          */
/* ---------------------------------------------------------------- */
static void trace(const scene *S, ray_t initial, uint32_t *rng, float out[4]) {
    const sg_settings *st = S->s;
    ray_t ray = initial;
    v3 throughput = V(1, 1, 1);
    v3 radiance = V(0, 0, 0);
    v3 backdrop = V(0, 0, 0);
    float previous_pdf = 0.0f;
    ray_t previous_vertex = initial;
    uint32_t depth = 0, null_crossings = 0;
    int point_gained = 0;
    float ring_cap = 1.0e30f;
    v3 ring_base = V(0, 0, 0);
    uint32_t shine_body = MISS;
    for (;;) {
        EV(vertices);
        hit_t hit = closest_hit(S, ray);
        float disc_scale = 1.0f;
        if (depth == 0u && null_crossings == 0u && st->background[3] > 0.0f)
            hit = point_disc_hit(S, ray, hit, &disc_scale, rng);
        ring_hit_t ring = closest_ring(S, ray, hit.distance);
        /* Host air and camera air (pathtrace.wgsl:1387-1414) are inert:
         * atmo_params.w < 0.5 for every frame the oracle accepts. */
        if (ring.index != MISS) {
            EV(ring_events);
            const sg_sphere *planet = &S->b[ring.index];
            if (depth == 0u && !point_gained && st->background[3] > 0.0f) {
                point_gained = 1;
                throughput = vmul(throughput, point_gain(S, planet->radius * planet->ring_params[0], ring.distance));
            }
            v3 n = b_pole(S, ring.index);
            optics_t optics = ring_optics(S, ring.index, ring.point);
            float mu_out = vdot(vneg(ray.dir), n);
            float transmission = ring_transmission(S, ray, ring);
            float scatter_probability = one_minus_exp(optics.tau / maxf_(fabsf(mu_out), 1.0e-7f));
            float bsdf_pdf = scatter_probability / (4.0f * PI_F);
            int last_vertex = depth + 1u == st->counts[3];
            float ring_mis = 1.0f;
            if (shine_body == ring.index && null_crossings == 0u) {
                float cos_ring = maxf_(fabsf(vdot(ray.dir, n)), 1.0e-6f);
                float shine_pdf = ring.distance * ring.distance / (ring_area(S, ring.index) * cos_ring);
                ring_mis = power_weight(previous_pdf, shine_pdf);
            }
            shine_body = MISS;
            float unshadowed = 0.0f, direct = 0.0f;
            uint32_t count = light_count(S);
            for (uint32_t slot = 0; slot < count; slot++) {
                uint32_t i = light_index(S, slot);
                if (b_emissive(S, i) < 0.5f || optics.tau == 0.0f) continue;
                ray_t origin = {ring.point, n, ring.index};
                light_sample light = sample_light(S, origin, i, rng);
                float mu_in = vdot(light.dir, n);
                float visibility = light_visibility(S, ring_origin(S, ring, light.dir), i);
                float weight = power_weight(light.pdf, bsdf_pdf);
                if (last_vertex) weight = 1.0f;
                v3 lit = vmul(vmulv(vmulv(throughput, ring_bsdf(optics, mu_out, mu_in)), b_color(S, i)),
                              fabsf(mu_in) / light.pdf);
                radiance = vadd(radiance, vmul(lit, visibility * weight * ring_mis));
                unshadowed += lum(lit);
                direct += lum(lit) * visibility;
            }
            if (rnd(S, rng) < transmission) {
                ray = ring_origin(S, ring, ray.dir);
                null_crossings += 1u;
                if (null_crossings > st->counts[0]) break;
                continue;
            }
            if (last_vertex || scatter_probability == 0.0f) break;
            if (ring_cap > 1.0e29f) {
                ring_cap = maxf_(direct, RING_INDIRECT_CAP * unshadowed);
                ring_base = radiance;
            }
            float z = 1.0f - 2.0f * rnd(S, rng);
            float phi = TAU_F * rnd(S, rng);
            float radial = sqrtf(maxf_(0.0f, 1.0f - z * z));
            v3 direction = basis_direction(n, radial * cosf(phi), radial * sinf(phi), z);
            throughput = vmul(vmulv(throughput, ring_bsdf(optics, mu_out, z)), fabsf(z) / bsdf_pdf);
            previous_pdf = bsdf_pdf;
            ray = ring_origin(S, ring, direction);
            previous_vertex = ray;
            depth += 1u;
            null_crossings = 0u;
            if (depth >= 3u) {
                float survival = clampf_(maxf_(throughput.x, maxf_(throughput.y, throughput.z)), 0.05f, 0.95f);
                if (rnd(S, rng) >= survival) break;
                throughput = vdivs(throughput, survival);
            }
            continue;
        }
        if (hit.index == MISS) {
            /* environment(): the catalogue is empty; milky_way(): no map is
             * bound, so both contribute zero radiance (pathtrace.wgsl:1494-1508). */
            break;
        }
        /* hit.index < LOCAL_BASE: the landscape is off. */
        uint32_t bi = hit.index;
        throughput = vmul(throughput, disc_scale);
        if (b_emissive(S, bi) > 0.5f) {
            float weight = 1.0f;
            if (depth > 0u) {
                float light_pdf = 1.0f / (TAU_F * cone_width(S, previous_vertex, hit.index));
                weight = power_weight(previous_pdf, light_pdf);
            }
            radiance = vadd(radiance, vmul(vmulv(throughput, b_color(S, bi)), weight));
            break;
        }
        EV(surface_events);
        if (depth == 0u && !point_gained && st->background[3] > 0.0f) {
            point_gained = 1;
            float extent = S->b[bi].radius * maxf_(1.0f, S->b[bi].ring_params[0]);
            throughput = vmul(throughput, point_gain(S, extent, hit.distance));
        }
        v3 normal = hit.normal;
        ray_t outgoing;
        outgoing.offset = vmul(normal, S->b[bi].radius * (1.0f + 2.0e-6f));
        outgoing.dir = normal;
        outgoing.anchor = hit.index;
        v3 direct_light = V(0, 0, 0);
        int last_vertex = depth + 1u == st->counts[3];
        uint32_t count = light_count(S);
        for (uint32_t slot = 0; slot < count; slot++) {
            uint32_t i = light_index(S, slot);
            if (b_emissive(S, i) < 0.5f) continue;
            light_sample sample = sample_light(S, outgoing, i, rng);
            float cosine = maxf_(vdot(normal, sample.dir), 0.0f);
            if (cosine <= 0.0f) continue;
            outgoing.dir = sample.dir;
            float visibility = light_visibility(S, outgoing, i);
            if (visibility > 0.0f) {
                float bsdf_pdf = cosine / PI_F;
                float weight = power_weight(sample.pdf, bsdf_pdf);
                if (last_vertex) weight = 1.0f;
                /* air_transmittance(...) == 1 without air. */
                direct_light = vadd(direct_light, vmul(b_color(S, i), bsdf_pdf * weight * visibility / sample.pdf));
            }
        }
        v3 albedo = surface_albedo(S, bi, normal);
        radiance = vadd(radiance, vmulv(vmulv(throughput, albedo), direct_light));
        shine_body = MISS;
        radiance = vadd(radiance, vmulv(vmulv(throughput, albedo),
                                        ringshine(S, hit.index, outgoing.offset, normal, last_vertex, rng)));
        shine_body = hit.index;
        if (last_vertex) break;
        float u = rnd(S, rng);
        float phi = TAU_F * rnd(S, rng);
        float cosine = sqrtf(1.0f - u);
        outgoing.dir = basis_direction(normal, sqrtf(u) * cosf(phi), sqrtf(u) * sinf(phi), cosine);
        previous_pdf = cosine / PI_F;
        throughput = vmulv(throughput, albedo);
        if (depth >= 2u) {
            float survival = clampf_(maxf_(throughput.x, maxf_(throughput.y, throughput.z)), 0.05f, 0.95f);
            if (rnd(S, rng) >= survival) break;
            throughput = vdivs(throughput, survival);
        }
        ray = outgoing;
        previous_vertex = outgoing;
        depth += 1u;
        null_crossings = 0u;
    }
    if (ring_cap < 1.0e29f) {
        v3 indirect = vsub(radiance, ring_base);
        float luminance = lum(indirect);
        if (luminance > ring_cap) radiance = vadd(ring_base, vmul(indirect, ring_cap / luminance));
    }
    out[0] = radiance.x;
    out[1] = radiance.y;
    out[2] = radiance.z;
    out[3] = lum(backdrop);
}

/* camera_direction: pathtrace.wgsl:1619-1626 */
static v3 camera_direction(const scene *S, uint32_t x, uint32_t y, uint32_t *rng) {
    float jx = rnd(S, rng);
    float jy = rnd(S, rng);
    float u = ((float)x + jx) / S->s->g.viewport[0];
    float v = ((float)y + jy) / S->s->g.viewport[1];
    float ndc_x = 2.0f * u - 1.0f;
    float ndc_y = 1.0f - 2.0f * v;
    float tangent = S->s->g.cam_forward[3];
    return vnormalize(V(ndc_x * tangent * S->s->g.viewport[3], ndc_y * tangent, -1.0f));
}

static int check_frame(const sg_settings *s) {
    if (!s) return SG_ERR_INVALID;
    if (s->g.atmo_params[3] >= 0.5f) return SG_ERR_INVALID;
    if (s->g.ground_north[3] != 0.0f) return SG_ERR_INVALID;
    if (s->counts[0] > SG_BODY_CAPACITY) return SG_ERR_CAPACITY;
    return SG_OK;
}

static void sample_pixel(const scene *S, uint32_t x, uint32_t y, uint32_t s, float out[4]) {
    uint32_t width = (uint32_t)S->s->g.viewport[0];
    uint32_t pixel = y * width + x;
    uint32_t rng = hash_u32(pixel ^ hash_u32(S->s->sampling[0] + s + 0x9e3779b9u));
    ray_t ray;
    ray.offset = V(0, 0, 0);
    ray.dir = camera_direction(S, x, y, &rng);
    ray.anchor = MISS;
    trace(S, ray, &rng, out);
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
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
    for (long k = 0; k < total; k++) {
#ifdef _OPENMP
        int tid = omp_get_thread_num();
#else
        int tid = 0;
#endif
        scene S = {settings, bodies, tables, per_thread ? &per_thread[tid] : NULL};
        uint32_t x = (uint32_t)(k % width);
        uint32_t y = y0 + (uint32_t)(k / width);
        uint32_t pixel = y * width + x;
        float sum[4] = {0, 0, 0, 0};
        /* The backdrop rgb sum stays zero: no Milky Way map is bound. */
        for (uint32_t s = 0; s < z; s++) {
            float r[4];
            if (S.ev) S.ev->samples++;
            sample_pixel(&S, x, y, s, r);
            for (int c = 0; c < 4; c++) sum[c] += r[c];
        }
        uint32_t old_count = settings->counts[1];
        uint32_t new_count = old_count + z;
        float mean[4], bmean[3];
        for (int c = 0; c < 4; c++) mean[c] = sum[c] / (float)z;
        for (int c = 0; c < 3; c++) bmean[c] = 0.0f / (float)z;
        if (old_count > 0u) {
            float w = (float)z / (float)new_count;
            for (int c = 0; c < 4; c++) {
                float old = accumulation[4 * pixel + c];
                mean[c] = old + (mean[c] - old) * w;
            }
            for (int c = 0; c < 3; c++) {
                float old = backdrop[4 * pixel + c];
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

int oracle_trace_sample(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                        uint32_t x, uint32_t y, uint32_t s, float out[4]) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL};
    sample_pixel(&S, x, y, s, out);
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
    scene S = {settings, bodies, tables, NULL};
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
    scene S = {settings, bodies, tables, NULL};
    for (uint32_t i = 0; i < n; i++) out[i] = light_visibility(&S, to_ray(&rays[i]), lights[i]);
    return SG_OK;
}

int oracle_reference_visibility(const sg_settings *settings, const sg_sphere *bodies, const oracle_tables *tables,
                                const sg_ray *rays, const uint32_t *lights, uint32_t n, float *out) {
    int status = check_frame(settings);
    if (status != SG_OK) return status;
    scene S = {settings, bodies, tables, NULL};
    for (uint32_t k = 0; k < n; k++) {
        ray_t ray = to_ray(&rays[k]);
        hit_t surface = closest_hit(&S, ray);
        if (surface.index != lights[k]) { out[k] = 0.0f; continue; }
        float transmission = 1.0f;
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
    scene S = {settings, bodies, tables, NULL};
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
    float energy = expf(-optics.tau / mu);
    for (uint32_t i = 0; i < steps; i++) {
        float mi = ((float)i + 0.5f) / (float)steps;
        v3 sum = vadd(ring_bsdf(optics, mu, mi), ring_bsdf(optics, mu, -mi));
        energy += sum.x * (TAU_F * mi / (float)steps);
    }
    return energy;
}

int oracle_sample_light(const sg_settings *settings, const sg_sphere *bodies, const sg_ray *ray,
                        uint32_t light, uint32_t *rng, float direction[3], float *pdf) {
    scene S = {settings, bodies, NULL, NULL};
    light_sample ls = sample_light(&S, to_ray(ray), light, rng);
    direction[0] = ls.dir.x;
    direction[1] = ls.dir.y;
    direction[2] = ls.dir.z;
    *pdf = ls.pdf;
    return SG_OK;
}

uint32_t oracle_hash(uint32_t value) { return hash_u32(value); }
float oracle_random(uint32_t *state) {
    scene S = {NULL, NULL, NULL, NULL};
    return rnd(&S, state);
}
