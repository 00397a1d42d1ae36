/*
 * stargaze_b200.h — C ABI of the B200 path-tracing integrator.
 *
 * Drop-in boundary for the wgpu compute pass that stargaze builds in
 * `PathTracer::new_with_guided_ground` and drives from `PathTracer::encode`
 * (src/pathtracer.rs:305-671, :789-1009). Scene buffers keep the reference's
 * byte layouts, so a caller that already packs `renderer::Frame` hands the
 * same bytes across this boundary.
 *
 * Conventions
 *   - Every entry point returns an `int` status: SG_OK (0) or a negative
 *     SG_ERR_* code. Nothing aborts the process; the reference's `assert!`
 *     panics (src/pathtracer.rs:795-800, :279-282) become status codes.
 *   - The library owns all device memory of a context. Host pointers passed
 *     in are borrowed for the duration of the call only.
 *   - One context per thread; calls on one context are not thread-safe.
 *   - `stream` arguments are `cudaStream_t` values passed as `void*`
 *     (NULL = legacy default stream).
 */
#ifndef STARGAZE_B200_H
#define STARGAZE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SG_API __attribute__((visibility("default")))
#else
#define SG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status codes                                                        */
/* ------------------------------------------------------------------ */
#define SG_OK 0
#define SG_ERR_INVALID -1   /* bad argument, size or pointer            */
#define SG_ERR_CAPACITY -2  /* body / primitive / table capacity         */
#define SG_ERR_CUDA -3      /* a CUDA runtime call failed                */
#define SG_ERR_OOM -4       /* device allocation failed                  */
#define SG_ERR_STATE -5     /* call not valid in the context's state     */
#define SG_ERR_TIMEOUT -6   /* a bounded device loop gave up             */

/* Capacities of the reference (src/pathtracer.rs:21-22, src/ground.rs:8). */
#define SG_BODY_CAPACITY 256
#define SG_MAX_BATCH_SAMPLES 64
#define SG_GROUND_CAPACITY 256
/* 2^24: the f32 sample-weight limit (src/graphics.rs:11). */
#define SG_MAX_SAMPLES 16777216u
/* Extension: landscape primitives this library accepts per frame. The
 * reference caps the list at SG_GROUND_CAPACITY; nested group markers
 * (center.w < 0) turn a longer list into a bounding-volume hierarchy that
 * the reference's own traversal (ground.wgsl:167-178) walks. */
#define SG_PROP_CAPACITY 65536
/* Extension: terrain grids up to 4096 cells per side (the reference stops
 * at 2048, src/terrain.rs:20). */
#define SG_TERRAIN_MAX_CELLS 4096
/* Extension: radial optical-depth tables for rings (no reference
 * counterpart; the reference has only a scalar or banded profile). */
#define SG_RING_TABLE_SLOTS 8
#define SG_RING_TABLE_MAX_BINS 4096
/* Marker for "no body" in Ray.anchor / Hit.index (pathtrace.wgsl:60). */
#define SG_MISS 0xffffffffu
/* Local landscape ids (ground.wgsl:14, terrain.wgsl:23). */
#define SG_LOCAL_BASE 0x80000000u
#define SG_TERRAIN_ID 0x80100000u

/* ------------------------------------------------------------------ */
/* Scene layouts (byte-identical to the reference)                     */
/* ------------------------------------------------------------------ */

/* renderer::Globals, src/renderer.rs:15-31 / pathtrace.wgsl:5-18. 176 B. */
typedef struct sg_globals {
    float cam_right[4];
    float cam_up[4];
    float cam_forward[4];   /* w = tan(vertical fov / 2)                     */
    float viewport[4];      /* trace width, height, exposure, display aspect  */
    float atmo_center[4];   /* xyz host centre (AU), w host radius            */
    float atmo_rayleigh[4]; /* rgb Rayleigh (1/AU), w Mie                     */
    float atmo_params[4];   /* Mie g, scale height, top, host index + 1       */
    float ground_east[4];   /* w = observer height (m)                        */
    float ground_up[4];     /* w = host radius (m)                            */
    float ground_north[4];  /* w = host index + 1 (0 disables the landscape)  */
    uint32_t ground_counts[4]; /* props, terrain on, theme | log2 cells << 8,
                                  prop top (f32 bits)                         */
} sg_globals;

/* pathtracer::Settings, src/pathtracer.rs:46-52 / pathtrace.wgsl:19-25. 240 B. */
typedef struct sg_settings {
    sg_globals g;
    uint32_t counts[4];   /* bodies, samples so far, samples now, max vertices */
    uint32_t sampling[4]; /* x = noise seed + sequence                         */
    float background[4];  /* Milky Way brightness, map w, map h, point gain    */
    uint32_t lights[4];   /* first three emissive indices, emissive count      */
} sg_settings;

/* renderer::Sphere, src/renderer.rs:35-48 / pathtrace.wgsl:26-37 (Body). 160 B. */
typedef struct sg_sphere {
    float center[3];          /* high part of the telescope-space centre (AU) */
    float radius;             /* AU                                            */
    float color[3];           /* reflectance or emitted radiance               */
    float emissive;           /* >= 0.5 : star                                 */
    float center_low[4];      /* xyz residual centre, w mottle strength        */
    float ring_plane[4];      /* xyz unit pole, w inner radius / body radius   */
    float ring_params[4];     /* outer / body radius, tau, banded,
                                 w: extension, ring-table slot + 1 (0 = none)  */
    float ring_color[4];      /* rgb single-scattering albedo                  */
    float axis_x[4];          /* xyz body X axis, w surface style              */
    float axis_y[4];          /* xyz body Y axis, w pattern seed               */
    float surface_color[4];
    float surface_params[4];
} sg_sphere;

/* ground::Primitive, src/ground.rs / ground.wgsl:3-7. 48 B. */
typedef struct sg_primitive {
    float center[4]; /* xyz surface-frame metres, w kind (<0 group marker)  */
    float extent[4]; /* xyz half extents, w yaw or packed tumble angles     */
    float albedo[4]; /* rgb tint, w material kind                           */
} sg_primitive;

/* pathtracer::Options, src/pathtracer.rs:77-111 (same defaults). */
typedef struct sg_options {
    uint32_t noise_seed;        /* 0                                   */
    uint32_t samples_per_frame; /* 1                                   */
    uint32_t max_bounces;       /* 8                                   */
    uint32_t sample_limit;      /* SG_MAX_SAMPLES                      */
    float exposure;             /* 1.0 (display only)                  */
    int32_t auto_exposure;      /* 0   (display only)                  */
    float ev_bias;              /* 0.0 (display only)                  */
    float auto_key;             /* 0.25 (display only)                 */
    float auto_percentile;      /* 0.9 (display only)                  */
    float milky_way;            /* 4e-4 camera-only backdrop brightness */
} sg_options;

/* renderer::Frame, src/renderer.rs:50-56 (HUD labels are not part of it). */
typedef struct sg_frame {
    const sg_globals *globals;
    const sg_sphere *bodies;
    uint32_t n_bodies;
    const sg_primitive *ground;
    uint32_t n_ground;
    double scene_time;
} sg_frame;

/* WGSL Ray (pathtrace.wgsl:70-76): origin = bodies[anchor] centre + offset,
 * anchor == SG_MISS means the camera origin. 28 B. */
typedef struct sg_ray {
    float offset[3];
    float direction[3];
    uint32_t anchor;
} sg_ray;

/* WGSL Hit (pathtrace.wgsl:77-81). 20 B. */
typedef struct sg_hit {
    float distance;
    uint32_t index;
    float normal[3];
} sg_hit;

typedef struct sg_context sg_context;

/* ------------------------------------------------------------------ */
/* Lifecycle — PathTracer::new / resize / drop                         */
/* ------------------------------------------------------------------ */

/* Fill `options` with the reference defaults (Options::default,
 * src/pathtracer.rs:95-111). */
SG_API int sg_default_options(sg_options *options);

/* PathTracer::new (src/pathtracer.rs:292-302): allocate the accumulation
 * for a width x height trace on CUDA device `device`. `options` may be NULL
 * for the defaults. */
SG_API int sg_create(int device, uint32_t width, uint32_t height,
              const sg_options *options, sg_context **out);

SG_API int sg_destroy(sg_context *ctx);

/* PathTracer::resize (src/pathtracer.rs:673-741): a new size reallocates the
 * accumulation and resets the sample history but keeps the noise sequence;
 * an unchanged size is a no-op. */
SG_API int sg_resize(sg_context *ctx, uint32_t width, uint32_t height);

/* ------------------------------------------------------------------ */
/* Progressive rendering — PathTracer::prepare_frame / set_quality /   */
/* encode / samples / needs_redraw                                     */
/* ------------------------------------------------------------------ */

/* PathTracer::prepare_frame (src/pathtracer.rs:756-759): update the
 * history key; *fresh = 1 when the accumulation was reset. */
SG_API int sg_prepare_frame(sg_context *ctx, const sg_frame *frame, int *fresh);

/* PathTracer::set_quality (src/pathtracer.rs:761-773). */
SG_API int sg_set_quality(sg_context *ctx, uint32_t samples, uint32_t bounces,
                   uint32_t limit);

/* Replace the whole option block (the reference's tests assign
 * `tracer.options` fields directly). Transport-relevant changes reset the
 * accumulation on the next encode through the history key. */
SG_API int sg_set_options(sg_context *ctx, const sg_options *options);
SG_API int sg_get_options(const sg_context *ctx, sg_options *options);

/* PathTracer::encode (src/pathtracer.rs:789-1009): validate capacities,
 * update the history, clamp the batch to SG_MAX_BATCH_SAMPLES and the
 * sample limit, upload the frame and enqueue the trace kernel on `stream`.
 * The call returns once the work is enqueued. */
SG_API int sg_encode(sg_context *ctx, const sg_frame *frame, void *stream);

/* History counters (PathTracer::samples, src/pathtracer.rs:742-744;
 * History::sequence, :166-171). */
SG_API int sg_get_samples(const sg_context *ctx, uint32_t *samples,
                   uint32_t *sequence);

/* PathTracer::needs_redraw (src/pathtracer.rs:749-752). */
SG_API int sg_needs_redraw(const sg_context *ctx, int *redraw);

SG_API int sg_get_size(const sg_context *ctx, uint32_t *width, uint32_t *height);

/* Read the running-mean accumulation: width*height float4 (rgb radiance,
 * w backdrop luminance), the buffer pathtracer_tests.rs:160-182 reads back.
 * `dst_on_device` selects a device or host destination; the call
 * synchronises `stream` before returning. */
SG_API int sg_read_accumulation(sg_context *ctx, float *dst, int dst_on_device,
                         void *stream);

/* Read the backdrop accumulation (binding 7): width*height float4. */
SG_API int sg_read_backdrop(sg_context *ctx, float *dst, int dst_on_device,
                     void *stream);

/* Resume support: restore an accumulation (width*height float4 means) with
 * its sample count and noise sequence. */
SG_API int sg_set_accumulation(sg_context *ctx, const float *src, int src_on_device,
                        uint32_t samples, uint32_t sequence, void *stream);

/* Device pointer of the accumulation (width*height float4), valid until the
 * next sg_resize / sg_destroy. */
SG_API int sg_accumulation_device_ptr(sg_context *ctx, void **ptr);

/* ------------------------------------------------------------------ */
/* Extension tables                                                    */
/* ------------------------------------------------------------------ */

/* Radial optical-depth profile for ring-table slot `slot`
 * (0 <= slot < SG_RING_TABLE_SLOTS). A body with ring_params.w == slot + 1
 * takes tau = ring_params.y * table[min(floor(x * bins), bins - 1)] at
 * normalised ring radius x, and its albedo from ring_color. Uploading bumps
 * the history key. No reference counterpart: rings.wgsl:50-81 has only the
 * scalar and banded profiles. */
SG_API int sg_upload_ring_profile(sg_context *ctx, uint32_t slot, const float *tau,
                           uint32_t bins);

/* Heightfield for the local landscape: `data` is the reference's
 * `terrain::Terrain::data` vector (src/terrain.rs:781-838) for a grid of
 * `cells` cells per side (power of two, 2..SG_TERRAIN_MAX_CELLS):
 * (cells+1)^2 heights, then (cells <= 1024 only) x and z derivatives, then
 * (min, max) per quadtree node in breadth-first order; `n_floats` is that
 * length, or that length plus the basalt elevation atlas
 * (`volcano::detail()`, src/volcano.rs:36-96), which the reference writes
 * at DETAIL_OFFSET, right after the geometry cache, and which basalt ground
 * (theme 4) shades from. The device appends the geometry cache of
 * cache_terrain_geometry (terrain.wgsl:242-285) on the next encode and
 * whenever the host radius (ground_up.w) changes. Frames with
 * ground_counts.y != 0 need an uploaded terrain. Uploading bumps the
 * history key. Replaces the ground buffer writes of src/pathtracer.rs:914-945. */
SG_API int sg_upload_terrain(sg_context *ctx, const float *data, size_t n_floats,
                             uint32_t cells);

/* Extension (no reference counterpart): a width x height scalar albedo map
 * over the surface frame; texel (i, j) covers x in
 * [-extent + 2*extent*i/width, ...) and likewise z, nearest-texel lookup.
 * When present it replaces the theme floor of the host ground and terrain
 * (ground.wgsl:601-610). width = 0 removes it. Bumps the history key. */
SG_API int sg_upload_albedo_map(sg_context *ctx, const float *albedo,
                                uint32_t width, uint32_t height,
                                float extent_m);

/* ------------------------------------------------------------------ */
/* Geometric queries (the reference's WGSL probe entry points)         */
/* ------------------------------------------------------------------ */

/* closest_hit over the frame (pathtrace.wgsl:173-185) for `n` rays.
 * rays/hits live on the device when `on_device`, else on the host. */
SG_API int sg_closest_hit(sg_context *ctx, const sg_frame *frame, const sg_ray *rays,
                   uint32_t n, sg_hit *hits, int on_device, void *stream);

/* light_visibility (rings.wgsl:90-115) of light body `lights[i]` along
 * rays[i]; out[i] in [0, 1]. */
SG_API int sg_light_visibility(sg_context *ctx, const sg_frame *frame,
                        const sg_ray *rays, const uint32_t *lights, uint32_t n,
                        float *out, int on_device, void *stream);

/* ring_hit of body `body` along rays[i] (rings.wgsl:8-34): out[4*i..] =
 * (distance, radius / body radius, ring_transmission, hit ? 1 : 0). */
SG_API int sg_ring_probe(sg_context *ctx, const sg_frame *frame, const sg_ray *rays,
                  uint32_t body, uint32_t n, float *out, int on_device,
                  void *stream);

/* terrain_hit in the surface frame (the terrain_probe entry point of
 * src/ground_tests.rs:700-705): rays[6*i..] = (origin xyz in metres,
 * direction xyz); out[4*i..] = (normal xyz, distance), distance 1e30 on a
 * miss. Uses the uploaded terrain, cached for the frame's host radius. */
SG_API int sg_terrain_probe(sg_context *ctx, const sg_frame *frame,
                            const float *rays, uint32_t n, float *out,
                            int on_device, void *stream);

/* closest_hit without device allocation. No counterpart in the reference.
 * For callers that cannot let the library allocate device memory at query
 * time: a host application that gives the whole device to its own
 * allocator or memory pool, where a library cudaMalloc fails or splits the
 * pool, and latency-bound callers, for which cudaMalloc synchronises the
 * device. The results equal sg_closest_hit's with FP64 sites off (this
 * entry point has no context, so it always runs the reference's f32
 * arithmetic). Unlike it, this call needs no
 * context and stages the frame's bodies, the rays and the hits in one
 * fixed device array of SG_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until the process exits.
 *   - rays and hits live in host memory; n <= SG_NOALLOC_MAX_RAYS, larger
 *     queries fail with SG_ERR_CAPACITY (split them);
 *   - frames with a local landscape (ground_north.w != 0) need a context
 *     and fail with SG_ERR_INVALID: use sg_closest_hit;
 *   - the first call on a device looks up the array's device address; make
 *     it before any stream capture. The address is kept for the life of the
 *     process: after cudaDeviceReset on that device, reload the library
 *     before calling this again;
 *   - every call on a device shares the array, so calls whose work
 *     overlaps on the GPU (other host threads, other streams) race;
 *   - errors are reported by sg_last_error(NULL).
 * Synchronises `stream` before returning. */
#define SG_NOALLOC_MAX_RAYS 65536u
#define SG_NOALLOC_SCRATCH_BYTES (4u << 20)
SG_API int sg_closest_hit_noalloc(int device, const sg_frame *frame, const sg_ray *rays,
                                  uint32_t n, sg_hit *hits, void *stream);

/* Energy of the ring slab BSDF (ring_tests.rs:352-413 probe): unscattered
 * transmission plus the cosine-weighted integral of ring_bsdf over both
 * hemispheres at outgoing cosine `mu`, midpoint rule with `steps` bins. */
SG_API int sg_ring_energy(sg_context *ctx, float albedo, float tau, float mu,
                   uint32_t steps, float *energy);

/* Extension (no reference counterpart): evaluate the three precision-
 * critical sites in FP64 from the same f32 inputs — the ring-plane
 * intersection (rings.wgsl:8-34), the host-sphere intersection of the local
 * landscape (ground.wgsl:138-158) and the 5 mm bounce offset with its
 * reprojection (ground.wgsl:649-662). Off by default, where the library
 * follows the reference's f32 arithmetic bit for bit. Changing it resets the
 * accumulation on the next encode. */
SG_API int sg_set_fp64_sites(sg_context *ctx, int enable);

/* The guided ground sampler: `guided` of PathTracer::new_with_guided_ground
 * (src/pathtracer.rs:305-312; the sampler is src/guided_ground.rs:14-79).
 * In frames with host air, a camera ray's local surface picks a reflecting
 * body (sample_reflector) and draws half of its continuations toward it,
 * weighting next-event and continuation by the full mixture density. Off by
 * default (the reference's plain constructor); the reference's app turns it
 * on. Changing it resets the accumulation on the next encode. */
SG_API int sg_set_guided_ground(sg_context *ctx, int enable);

/* Ringshine: the next-event estimation of a ringed planet's own sunlit
 * rings onto its surface (ringshine, pathtrace.wgsl:1248-1296, called from
 * trace at :1567-1571, with the MIS of continuations that reach the rings at
 * :1424-1430). On by default, as in the reference. Off reproduces the
 * integrator as it stood before ringshine was added, the one the
 * reference's published benchmark images were rendered with
 * (benchmarks/optimizations/rx7600xt-2026-10-04/, benchmarks/m4pro-2026-10-15/).
 * Changing it resets the accumulation on the next encode. */
SG_API int sg_set_ringshine(sg_context *ctx, int enable);

/* Extension (no reference counterpart; the reference renders forward only):
 * vertex checkpoints for sg_backward, the alternative to replaying every
 * path from its noise key. With `every` > 0, each wavefront sg_encode of an
 * accumulation stores a path's whole state (SG_CHECKPOINT_BYTES) whenever a
 * scatter brings its depth to a multiple of `every`, and every sample's
 * radiance (16 B per sample and pixel, for the first `max_samples` samples
 * of the accumulation). sg_backward then replays each sample only up to its
 * first checkpoint and every later segment from its record, in parallel,
 * with the path's total known, so nothing is deferred or replayed twice.
 * An `every` of at least the bounce limit stores the radiance alone (no
 * record buffer is allocated): the backward then replays whole paths, once
 * each, with every weight known.
 * Samples whose ring-indirect cap binds, or whose records did not fit
 * `record_bytes` (0: half the free device memory at the first encode), are
 * replayed from their noise key as without checkpoints. Frames with host
 * air, procedural styles or a sky backdrop, the megakernel integrator and
 * sg_encode_counted store none (their samples replay). `every` = 0 (the
 * default) turns checkpointing off and frees the buffers; a change resets
 * the accumulation on the next encode. */
#define SG_CHECKPOINT_BYTES 128u
SG_API int sg_set_checkpoints(sg_context *ctx, uint32_t every, uint32_t max_samples, uint64_t record_bytes);

/* Device memory the checkpoints of the current accumulation hold (totals
 * plus stored records), the records stored, and the records that did not
 * fit the budget. Any pointer may be NULL. Synchronises the device. */
SG_API int sg_get_checkpoint_stats(sg_context *ctx, uint64_t *device_bytes, uint64_t *records, uint64_t *dropped);

/* Extension (no reference counterpart; the reference has one WGSL compute
 * pass, pathtrace.wgsl:1645-1675): which CUDA integrator sg_encode runs.
 *   SG_INTEGRATOR_MEGAKERNEL  one thread per pixel walks every path of the
 *                             dispatch to its end;
 *   SG_INTEGRATOR_WAVEFRONT   (default) paths live in a pool of `pool_paths`
 *                             slots in device memory (0: 16 Mi, about 280 B
 *                             each, or the dispatch's sample count if that is
 *                             smaller) and advance one vertex per stage
 *                             iteration through extend / ring / surface
 *                             kernels over compacted queues.
 * Both run the same per-path code on the same random sequences; their
 * accumulations agree to a few ulps (the compiler fuses shading multiply-
 * adds differently in the two kernels). The wavefront allocates its pool
 * and a per-sample radiance buffer (16 B per pixel and sample, up to
 * 2.25 GiB; larger dispatches run in sample chunks) on first use, and its
 * sg_encode returns once the dispatch's stages have drained (it reads a
 * 32-byte counter back every few iterations). sg_encode_counted always runs
 * the megakernel. The choice does not reset the accumulation. */
#define SG_INTEGRATOR_MEGAKERNEL 0
#define SG_INTEGRATOR_WAVEFRONT 1
#define SG_WAVE_MAX_POOL (1u << 26)
SG_API int sg_set_integrator(sg_context *ctx, int integrator, uint32_t pool_paths);

/* The integrator in use, the wavefront pool of the last dispatch and the
 * stage iterations it ran (0 for the megakernel). Any pointer may be NULL. */
SG_API int sg_get_integrator(const sg_context *ctx, int *integrator, uint32_t *pool_paths,
                             uint32_t *iterations);

/* The camera-only sky backdrop of primary misses (pathtrace.wgsl:268-334,
 * :1494-1508), bound in the reference as the `catalogue`, `sky_cells` and
 * `milky_way` buffers (src/pathtracer.rs:319-368, the tables built by
 * src/stars.rs:152-201 and src/sky.rs:103-119).
 *   sg_upload_catalogue: `n` stars of 8 floats (direction xyz, sin^2 of the
 *     angular radius, radiance rgb, unused) and the 256 x 128 cell table:
 *     32,769 non-decreasing offsets (the first 0, the last the index count)
 *     followed by the star indices of each cell. n = 0 removes it.
 *   sg_upload_milky_way: width x height texels of 10-bit linear RGB
 *     (r | g << 10 | b << 20), scaled by options.milky_way. A zero size
 *     removes it.
 * Unscattered camera paths then see the catalogue's discs and the Milky Way
 * through their ring transmissions; the Milky Way is also accumulated apart
 * (sg_read_backdrop) and its luminance is the accumulation's w channel.
 * Uploads reset the accumulation. sg_backward rejects frames with a sky. */
SG_API int sg_upload_catalogue(sg_context *ctx, const float *stars, uint32_t n, const uint32_t *cells,
                               uint32_t n_cells);
SG_API int sg_upload_milky_way(sg_context *ctx, const uint32_t *texels, uint32_t width, uint32_t height);

/* ------------------------------------------------------------------ */
/* Display without a graphics API                                      */
/* ------------------------------------------------------------------ */

/* The reference's display pass (display.wgsl:69-97, drawn by
 * PathTracer::display, src/pathtracer.rs:1010-1014) into a device buffer
 * instead of a swapchain or texture: each of width x height output pixels
 * samples the accumulation bilinearly at its centre (any output size: the
 * reference upscales the trace resolution to the window), applies the
 * exposure in stops — the eased automatic value when options.auto_exposure
 * is on, else options.exposure — plus options.ev_bias, limits the Milky Way
 * backdrop layer and maps through the ACES curve.
 *   SG_DISPLAY_RGBA8_SRGB  4 bytes per pixel, R G B A, sRGB-encoded as a
 *                          Rgba8UnormSrgb target stores it (the format of
 *                          the reference's headless PNG, src/headless.rs:13)
 *   SG_DISPLAY_RGBA32F     4 floats per pixel, linear (the reference's
 *                          Rgba32Float test targets)
 * `out` lives on the device when `on_device`, else on the host (the call
 * then synchronises `stream`). */
#define SG_DISPLAY_RGBA8_SRGB 0
#define SG_DISPLAY_RGBA32F 1
SG_API int sg_display(sg_context *ctx, uint32_t width, uint32_t height, int format, void *out,
                      int on_device, void *stream);

/* The exposure the display uses now: the eased automatic value when
 * options.auto_exposure is on (metered by every sg_encode, including ones
 * that add no sample, as PathTracer::encode does, src/pathtracer.rs:980-
 * 1000), else options.exposure. Synchronises `stream`. */
SG_API int sg_get_exposure(sg_context *ctx, float *exposure, void *stream);

/* PathTracer::set_exposure_controls (src/pathtracer.rs:777-781): automatic
 * metering on or off and the exposure compensation in stops. Display only:
 * the accumulation is kept; the 60-frame settle of sg_needs_redraw
 * restarts. */
SG_API int sg_set_exposure_controls(sg_context *ctx, int automatic, float bias);

/* Extension (measurement): with timing on, every wavefront stage launch is
 * bracketed by CUDA events and sg_encode waits for the dispatch to finish;
 * sg_get_stage_times then gives the milliseconds of the last timed
 * dispatch spent in ms[0] extend, ms[1] ring, ms[2] surface, ms[3] resolve,
 * ms[4] between stages (launch gaps and host checks) and ms[5] finishing
 * the last few paths of each sample chunk in one launch. */
#define SG_STAGE_COUNT 6
SG_API int sg_set_stage_timing(sg_context *ctx, int enable);
SG_API int sg_get_stage_times(const sg_context *ctx, float *ms);

/* ------------------------------------------------------------------ */
/* Path-replay adjoint (extension: the reference renders forward only) */
/* ------------------------------------------------------------------ */

#define SG_TAPE_RANGES 16

/* What the forward saves for the backward: the noise keys of every sample
 * behind the current accumulation — runs of consecutive keys, a sample's
 * key being the dispatch's sampling.x plus its index in the batch — and a
 * hash of the history key (frame, options, uploaded tables) they were
 * rendered with. The backward replays exactly these samples. */
typedef struct sg_tape {
    uint32_t width, height;
    uint32_t samples;                /* samples behind the accumulation      */
    uint32_t n_ranges;
    uint32_t first[SG_TAPE_RANGES];  /* first noise key of each run          */
    uint32_t count[SG_TAPE_RANGES];  /* samples of each run                  */
    uint64_t history_hash;
} sg_tape;

/* Gradient destinations of sg_backward; a NULL pointer skips that block.
 * All values are d loss / d parameter, summed over the image. */
typedef struct sg_gradients {
    /* SG_RING_TABLE_SLOTS * SG_RING_TABLE_MAX_BINS, slot-major: the ring
     * optical-depth table values of sg_upload_ring_profile. */
    float *ring_tau;
    /* n_bodies * 3: sg_sphere.ring_color (single-scattering albedo). */
    float *ring_albedo;
    /* n_bodies * 3: sg_sphere.color — albedo of a surface, emitted radiance
     * of an emitter (luminosity follows by the chain rule). */
    float *body_color;
    /* map width * height: the texels of sg_upload_albedo_map. */
    float *albedo_map;
    /* out: derivative entries dropped because a path's list was full (a
     * path with more than 32 throughput factors); 0 in normal scenes. */
    uint64_t dropped;
} sg_gradients;

/* The tape of the current accumulation (the forward's saved state, the
 * torch.autograd.Function contract's ctx.save_for_backward). SG_ERR_STATE
 * when the accumulation cannot be replayed: restored by
 * sg_set_accumulation, or mixing more than SG_TAPE_RANGES key runs. */
SG_API int sg_get_tape(const sg_context *ctx, sg_tape *tape);

/* Backward pass: replay every sample of `tape` on `frame` (which must hash
 * to the tape's history key: same frame, options and tables as the forward)
 * and accumulate the gradient of a loss with d loss / d image =
 * `dl_dimage` (width*height float4, the w channel ignored) into `grads`.
 * Sampling is detached (the estimator's random decisions are held fixed),
 * so the result is an unbiased estimate of the gradient of the expected
 * image. `on_device` applies to dl_dimage and to every gradient pointer.
 * The accumulation is not modified. Synchronises `stream`. With the
 * wavefront integrator (the default) the replay runs in the same stages as
 * the forward, over a pool of up to 16 Mi paths (pool_paths of
 * sg_set_integrator when set) holding about 1.1 KB of device memory each,
 * allocated on first use; with the megakernel, one thread per pixel.
 * SG_ERR_STATE for frames whose radiance this adjoint does not
 * differentiate: a sky backdrop (catalogue or panorama bound), host air
 * (atmo_params.w >= 0.5) or a body with a procedural surface style
 * (axis_x.w >= 0.5). */
SG_API int sg_backward(sg_context *ctx, const sg_frame *frame, const sg_tape *tape,
                       const float *dl_dimage, int on_device, sg_gradients *grads,
                       void *stream);

/* ------------------------------------------------------------------ */
/* Diagnostics                                                         */
/* ------------------------------------------------------------------ */

/* Last error message of the context (or of the library when ctx is NULL). */
SG_API const char *sg_last_error(const sg_context *ctx);
SG_API const char *sg_status_string(int status);
/* Number of integrator kernel launches issued by this context so far (one
 * per megakernel dispatch; three per wavefront iteration plus one resolve
 * per sample chunk). */
SG_API int sg_launch_count(const sg_context *ctx, uint64_t *launches);

/* sg_encode through the event-counting variant of the integrator kernel:
 * same image and history effect, plus per-dispatch event totals in
 * `events[SG_EVENT_COUNT]` (vertices, sphere tests, sphere hits, ring tests,
 * light samples, shadow rays, ring events, surface events, RNG draws,
 * terrain quadtree nodes expanded, terrain triangle tests, landscape
 * group-marker box tests, landscape primitive tests).
 * Synchronises `stream`. Used to model the algorithmic work of a launch. */
#define SG_EVENT_COUNT 13
SG_API int sg_encode_counted(sg_context *ctx, const sg_frame *frame,
                             void *stream, uint64_t *events);

/* Measure the FP32 FMA issue peak of `device`: an FMA-chain kernel over
 * every SM, timed with CUDA events. Returns FLOP/s (2 per FMA). */
SG_API int sg_measure_fp32_peak(int device, double *flops_per_second);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* STARGAZE_B200_H */
