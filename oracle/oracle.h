/*
 * oracle.h — CPU restatement of stargaze's progressive path-tracing
 * integrator (src/shaders/pathtrace.wgsl, src/shaders/rings.wgsl).
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA
 * integrator: only the test suite, the smoke check and the CPU-baseline leg
 * of the benchmark load it. The product path never calls it.
 *
 * Parity pin: the reference is Rust + WGSL executed by wgpu, which cannot be
 * built or run here (no Rust toolchain, no graphics stack). The restatement
 * is pinned against the reference's own analytic known-answer tests
 * (src/pathtracer_tests.rs, src/ring_tests.rs, src/ground_tests.rs), which
 * the test suite re-runs against this library.
 *
 * Arithmetic is IEEE f32 compiled with -ffp-contract=off, so + - * / sqrt
 * follow the WGSL expression order exactly; transcendental functions come
 * from the C library.
 */
#ifndef STARGAZE_ORACLE_H
#define STARGAZE_ORACLE_H

#include "../include/stargaze_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Extension tables the oracle shares with the CUDA path. */
typedef struct oracle_tables {
    const float *ring_tau[SG_RING_TABLE_SLOTS];
    uint32_t ring_bins[SG_RING_TABLE_SLOTS];
} oracle_tables;

/* Per-sample event counters (used to pin the CUDA event counts). */
typedef struct oracle_events {
    uint64_t samples;
    uint64_t vertices;       /* trace loop iterations                   */
    uint64_t sphere_tests;   /* sphere_hit_radius calls                 */
    uint64_t sphere_hits;    /* ... that returned a hit                 */
    uint64_t ring_tests;     /* ring_hit calls past the presence check  */
    uint64_t light_samples;  /* sample_light_stratum calls              */
    uint64_t shadow_rays;    /* light_visibility calls                  */
    uint64_t ring_events;    /* ring scattering / null vertices         */
    uint64_t surface_events; /* surface shading vertices                */
    uint64_t rng_draws;      /* random() calls                          */
} oracle_events;

/* One dispatch of the WGSL `main` entry point (pathtrace.wgsl:1645-1675)
 * over pixel rows [y0, y1): for each pixel, counts.z samples through
 * trace(), then the running-mean update of `accumulation` and `backdrop`
 * (width*height float4 each, read when counts.y > 0). Viewport size is
 * settings->g.viewport.xy. `threads` <= 0 uses all OpenMP threads. */
int oracle_dispatch(const sg_settings *settings, const sg_sphere *bodies,
                    const oracle_tables *tables, float *accumulation,
                    float *backdrop, uint32_t y0, uint32_t y1, int threads,
                    oracle_events *events);

/* One sample: trace() for pixel (x, y), sample index s of the dispatch.
 * out = (radiance rgb, backdrop luminance). */
int oracle_trace_sample(const sg_settings *settings, const sg_sphere *bodies,
                        const oracle_tables *tables, uint32_t x, uint32_t y,
                        uint32_t s, float out[4]);

/* closest_hit (pathtrace.wgsl:173-185) for n rays. */
int oracle_closest_hit(const sg_settings *settings, const sg_sphere *bodies,
                       const oracle_tables *tables, const sg_ray *rays,
                       uint32_t n, sg_hit *hits);

/* light_visibility (rings.wgsl:90-115). */
int oracle_light_visibility(const sg_settings *settings,
                            const sg_sphere *bodies,
                            const oracle_tables *tables, const sg_ray *rays,
                            const uint32_t *lights, uint32_t n, float *out);

/* Reference shadow test of ground_tests.rs:1064-1075: closest_hit must be
 * the light, then the product of ring transmissions before it. */
int oracle_reference_visibility(const sg_settings *settings,
                                const sg_sphere *bodies,
                                const oracle_tables *tables,
                                const sg_ray *rays, const uint32_t *lights,
                                uint32_t n, float *out);

/* ring_hit probe (ring_tests.rs:71-82): out[4i..] = (distance,
 * radius/body radius, ring_transmission, hit). */
int oracle_ring_probe(const sg_settings *settings, const sg_sphere *bodies,
                      const oracle_tables *tables, const sg_ray *rays,
                      uint32_t body, uint32_t n, float *out);

/* Ring slab energy probe (ring_tests.rs:365-377). */
float oracle_ring_energy(float albedo, float tau, float mu, uint32_t steps);

/* sample_light direction for a ray (used to build seeded shadow rays the way
 * ground_tests.rs:1086-1092 does). rng is advanced in place. */
int oracle_sample_light(const sg_settings *settings, const sg_sphere *bodies,
                        const sg_ray *ray, uint32_t light, uint32_t *rng,
                        float direction[3], float *pdf);

/* hash / random of pathtrace.wgsl:87-98, exported for RNG-stream checks. */
uint32_t oracle_hash(uint32_t value);
float oracle_random(uint32_t *state);

#ifdef __cplusplus
}
#endif

#endif
