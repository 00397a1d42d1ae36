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
 * (src/pathtracer_tests.rs, src/ring_tests.rs, src/ground_tests.rs,
 * src/planetshine_tests.rs), which the test suite re-runs against this
 * library. Landscape themes 3-5 and vegetation have no such tests outside
 * the reference's YAML scenes: their restatement is pinned by reading.
 *
 * Arithmetic is IEEE f32 compiled with -ffp-contract=off, so + - * / sqrt
 * follow the WGSL expression order exactly; transcendental functions come
 * from the C library (in double, rounded to f32, where the WGSL hashes
 * coordinates derived from them).
 */
#ifndef STARGAZE_ORACLE_H
#define STARGAZE_ORACLE_H

#include "../include/stargaze_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Scene data beyond the body table, shared with the CUDA path. */
typedef struct oracle_tables {
    const float *ring_tau[SG_RING_TABLE_SLOTS];
    uint32_t ring_bins[SG_RING_TABLE_SLOTS];
    /* Heightfield in the reference layout (src/shaders/terrain.wgsl:1-20):
     * heights, [x/z derivatives], min/max per quadtree node, node AABBs,
     * vertex cache. NULL disables terrain. The cache part is filled by
     * oracle_cache_terrain. */
    const float *terrain;
    uint32_t terrain_cells;
    /* Floats of the measured elevation atlas that follows the vertex cache
     * (basalt ground, volcano.wgsl); 0 without one. */
    uint32_t terrain_detail_floats;
    /* Landscape primitives of the frame (ground.wgsl:3-12). */
    const sg_primitive *ground;
    uint32_t n_ground;
    /* Extension: scalar albedo map over the surface frame, texel (i, j)
     * covers x, z in [-extent, extent]; NULL uses the theme floor. */
    const float *albedo_map;
    uint32_t map_width, map_height;
    float map_extent;
    /* Camera-only sky backdrop (pathtrace.wgsl:268-334): catalogue rows of
     * 8 floats (direction, sin^2 radius, radiance, unused) with the 256 x 128
     * cell table (32,769 offsets, then indices), and the RGB10 Milky Way
     * panorama (its size in settings.background.yz). NULL disables each. */
    const float *catalogue;
    uint32_t catalogue_n;
    const uint32_t *sky_cells;
    const uint32_t *milky_way;
    /* The guided ground sampler (src/guided_ground.rs:14-79) when nonzero. */
    uint32_t guided_ground;
    /* Nonzero leaves out ringshine (pathtrace.wgsl:1248-1296): no annulus
     * sample, no light samples from it and no MIS of continuations that hit
     * the rings. This is the integrator the reference's published benchmark
     * images were rendered with (their manifests predate ringshine). */
    uint32_t ringshine_off;
} oracle_tables;

/* Floats of the reference terrain layout for `cells` cells per side
 * (terrain.wgsl:6-20): everything up to and including the vertex cache. */
size_t oracle_terrain_floats(uint32_t cells);

/* cache_terrain_geometry (terrain.wgsl:242-285) for host radius
 * `radius_m`: fills the node AABBs and the vertex cache of `terrain`. */
int oracle_cache_terrain(float *terrain, uint32_t cells, float radius_m);

/* terrain_query (terrain.wgsl:152-234) in the surface frame: out =
 * (normal xyz, distance), distance 1e30 on a miss. */
int oracle_terrain_query(const sg_settings *settings, const oracle_tables *tables, const float o[3],
                         const float d[3], float limit, int occlusion, float out[4]);

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
    uint64_t terrain_nodes;  /* quadtree interior nodes expanded        */
    uint64_t terrain_triangles; /* terrain_triangle calls               */
    uint64_t prop_boxes;     /* group-marker bounding-box tests         */
    uint64_t prop_tests;     /* landscape primitive tests               */
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

/* Checker of the CUDA adjoint (an extension without reference
 * counterpart). A direction assigns a tangent to each material parameter
 * (NULL blocks are zero): per-bin ring-table values, ring albedo and body
 * colour (3 floats per body), albedo-map texels. */
typedef struct oracle_direction {
    const float *ring_tau[SG_RING_TABLE_SLOTS];
    const float *ring_albedo;
    const float *body_color;
    const float *albedo_map;
} oracle_direction;

/* Forward-mode derivative of the detached-sampling estimator: for pixel
 * rows [y0, y1) and the counts.z samples of the dispatch, adds the radiance
 * (primal, 4 floats per pixel) and its tangent along `direction` (tangent,
 * 4 floats per pixel, w unused) to the output sums. Sampling decisions,
 * pdfs, MIS weights and Russian-roulette survivals keep their values;
 * the ring-indirect cap is differentiated exactly. */
int oracle_tangent(const sg_settings *settings, const sg_sphere *bodies,
                   const oracle_tables *tables, const oracle_direction *direction,
                   float *primal, float *tangent, uint32_t y0, uint32_t y1,
                   int threads);

/* hash / random of pathtrace.wgsl:87-98, exported for RNG-stream checks. */
/* The surface sky cache of a frame with host air (terrain.wgsl:286-302):
 * 16 x 8 float4 texels, row-major by elevation. */
int oracle_sky_cache(const sg_settings *settings, const sg_sphere *bodies,
                     const oracle_tables *tables, float out[4 * 128]);

uint32_t oracle_hash(uint32_t value);
float oracle_random(uint32_t *state);

#ifdef __cplusplus
}
#endif

#endif
