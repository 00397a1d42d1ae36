// sg_internal.h — launch interface between the C-ABI host runtime and the
// CUDA kernels of the integrator.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/stargaze_b200.h"

namespace sg {

// Everything one integrator launch reads. Passed by value as a
// __grid_constant__ parameter (it lands in the constant bank).
struct TraceParams {
    sg_settings s;                           // 240 B, the WGSL `settings` uniform
    const float4 *bodies;                    // counts.x * 10 float4 (sg_sphere)
    const float *tables;                     // ring tables, slot-major
    uint32_t bins[SG_RING_TABLE_SLOTS];      // bins per slot (0 = empty)
    uint32_t table_stride;                   // floats between slots
    uint32_t staged_table_floats;            // floats staged into shared memory
    float4 *mean;                            // accumulation (running mean)
    float4 *sum;                             // compensated sum
    float4 *comp;                            // Kahan compensation
    uint32_t width, height;
    unsigned long long *events;              // optional event counters (9)
    // Local landscape (ground.wgsl, terrain.wgsl): heightfield in the
    // reference layout with its device-computed cache, props as 3 float4
    // (center, extent, albedo) each, optional scalar albedo map.
    const float *terrain;
    uint32_t terrain_cells;
    uint32_t terrain_detail_floats;  // basalt elevation atlas after the vertex cache
    const float4 *props;
    const float4 *prop_trig;  // 2 float4 per prop: (sin, cos) of x, y; z
    uint32_t n_props;
    const float *albedo_map;
    uint32_t map_width, map_height;
    float map_extent;
    uint32_t fp64_sites;  // ring plane, host sphere and 5 mm offset in FP64
    // Camera-only sky backdrop (pathtrace.wgsl:268-334): the star catalogue
    // (2 float4 per star: direction + sin^2 radius, radiance) with its
    // 256 x 128 cell table (32,769 offsets, then indices), and the Milky Way
    // panorama (RGB10 texels); `backdrop` receives its running mean.
    const float4 *catalogue;
    const uint32_t *sky_cells;
    uint32_t catalogue_n;
    const uint32_t *milky_way;
    uint32_t sky_on;  // catalogue or panorama bound (and the panorama's brightness > 0)
    float4 *backdrop;
    // Host air (atmo_params.w >= 0.5): its surface sky cache, 16 x 8 float4
    // texels (terrain.wgsl:286-302), built when an accumulation starts.
    uint32_t air_on;
    const float4 *sky_light;
    // The guided ground sampler (src/guided_ground.rs:14-79): depth-0 local
    // surfaces under air also propose directions toward a reflecting body.
    uint32_t guided_ground;
    // A body of the frame has a procedural surface style (axis_x.w >= 0.5).
    uint32_t styled;
    // Ringshine next-event estimation (pathtrace.wgsl:1248-1296) at ringed
    // bodies' surfaces; 0 leaves it out (sg_set_ringshine).
    uint32_t ringshine;
    // Per 16x16 pixel tile of the viewport: the bodies (x) and rings (y) a
    // camera ray of the tile can meet, by a conservative cone test
    // (launch_camera_cull). Camera rays skip the others' intersection
    // tests, which would miss. Null: test every body.
    const uint2 *camera_cull;
};

// The camera-ray cull masks of every 16x16 tile into `out` (tiles_x *
// tiles_y entries) for frames of at most 32 bodies.
cudaError_t launch_camera_cull(const TraceParams &p, uint2 *out, cudaStream_t stream);

// Geometry cache of the heightfield (cache_terrain_geometry,
// terrain.wgsl:242-285) for host radius `radius_m`, in place.
cudaError_t launch_terrain_cache(float *terrain, uint32_t cells, float radius_m, cudaStream_t stream);

// Floats of the full device terrain layout for `cells` cells per side.
size_t terrain_floats(uint32_t cells);
size_t terrain_source_floats(uint32_t cells);

constexpr int kEventCount = SG_EVENT_COUNT;

// Shared-memory bytes a launch with these parameters needs.
size_t trace_smem_bytes(const TraceParams &p);

// Sets the message sg_last_error(NULL) returns (entry points without a
// context report through it).
void set_library_error(const char *message);

cudaError_t launch_trace(const TraceParams &p, bool count_events, cudaStream_t stream);

// cache_surface_sky (terrain.wgsl:286-302) into `out` (128 float4): the
// in-scatter of 16 x 8 directions of the local sky, seen from the camera.
constexpr uint32_t kSkyCacheTexels = 128;
cudaError_t launch_sky_cache(const TraceParams &p, float4 *out, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Wavefront integrator (sg_wavefront.cu): the same per-path arithmetic as
// launch_trace, run as extend / ring / surface stages over queues
// of paths whose state lives in HBM, then an in-order per-pixel resolve.
// ---------------------------------------------------------------------------

// Counters of one iteration of the stage loop.
struct WaveCounters {
    uint32_t cont;     // paths the previous iteration's shade stages kept
    uint32_t unused;
    uint32_t ring;     // ring-queue entries extend wrote
    uint32_t surface;  // surface-queue entries extend wrote
    uint32_t next;     // first sample index (within the chunk) not taken yet
    uint32_t pad[3];
};
// Iteration t uses counter sets t and t + 1 (mod this) and clears t + 2.
constexpr uint32_t kWaveCounterSets = 8;

// How far the GPU has got through a stage loop: at its start, extend of
// iteration t writes (paths kept, next sample) to slot t % kProgressSlots of
// a ring in mapped host memory, and the host records done[t % ...] after
// the iteration. The host enqueues iterations ahead of the one it inspects,
// so the GPU does not wait for it between iterations.
constexpr uint32_t kProgressSlots = 8;
struct WaveProgress {
    uint2 *host = nullptr;    // mapped pinned memory, kProgressSlots slots
    uint2 *device = nullptr;  // its device address
    cudaEvent_t done[kProgressSlots] = {};
};
// Float4 planes of one path's state, and of one extend result.
constexpr uint32_t kWavePlanes = 7;
constexpr uint32_t kWaveHitPlanes = 3;

// Vertex checkpoints (sg_set_checkpoints): the forward stores a path's
// whole state each time a scatter brings its depth to a multiple of
// `every` (up to max_depth), and every sample's radiance before the ring
// cap with its checkpoint bits. The backward then replays each segment
// between checkpoints on its own instead of every path from its seed.
//   record r: kWavePlanes float4 of path state (the pool's planes), then
//             (pixel, sample, depth, 0) — `sample` indexes the accumulation;
//   totals[sample * pixels + pixel] = (radiance, bits): bit 0 the sample has
//             records, bit 1 it must be replayed from its seed (a record did
//             not fit, or its ring-indirect cap binds).
constexpr uint32_t kCheckpointVec4 = 8;
struct Checkpoints {
    float4 *records;          // capacity * kCheckpointVec4 float4
    uint32_t *count;          // records claimed (may exceed capacity)
    uint32_t capacity;
    float4 *totals;           // samples * pixels entries
    uint32_t samples;         // accumulation samples `totals` covers
    uint32_t sample_base;     // accumulation index of the dispatch's first sample
    uint32_t every;
    uint32_t max_depth;
};

struct WaveParams {
    float4 *state[2];         // kWavePlanes planes of `pool` float4 each
    float4 *hits;             // kWaveHitPlanes planes of `pool` float4
    uint32_t *ring_queue;     // `pool` path indices
    uint32_t *surface_queue;  // `pool` path indices
    WaveCounters *counters;   // kWaveCounterSets sets
    uint2 *progress;          // WaveProgress::device
    float4 *results;          // chunk_samples planes of width * height radiance samples
    float4 *totals;           // per-pixel running sums between chunks
    float4 *sky_results;      // as results, the backdrop of each sample (null: no sky)
    float4 *sky_totals;       // as totals, for the backdrop
    uint32_t pool;            // path slots
    uint32_t tiles_x, tiles_y;
    uint32_t chunk_first;     // first sample of the chunk within the dispatch
    uint32_t chunk_samples;   // samples of the chunk
    Checkpoints ck;           // vertex checkpoints of the forward (off: ck.records null)
};

// Bytes of the per-context wavefront buffers for `pool` path slots and
// results for `chunk_samples` samples of `pixels` pixels.
size_t wave_state_bytes(uint32_t pool);
size_t wave_result_bytes(uint32_t pixels, uint32_t chunk_samples);

// Optional per-stage timing of a wavefront dispatch: an event is recorded
// at every stage boundary; stage[k] names what runs from mark k to k + 1.
enum WaveStage : int { kStageExtend = 0, kStageRing, kStageSurface, kStageResolve, kStageGap, kStageFinish, kStageCount };
struct StageMarks {
    std::vector<cudaEvent_t> events;  // owned; grown on demand, reused
    std::vector<int> stage;
    size_t used = 0;
};

// What one wavefront dispatch ran.
struct WaveRun {
    uint32_t iterations = 0;  // stage iterations over all chunks
    uint32_t kernels = 0;     // kernel launches
};

// Runs the dispatch described by `p` (counts.z samples) in chunks of at
// most w.chunk_samples samples. It reads the GPU's progress (`progress`,
// w.progress its device ring) a few iterations behind the last one it
// enqueued to decide whether the chunk has drained, so it returns once the
// GPU has nearly finished. With `marks`, events bracket every stage.
cudaError_t launch_wavefront(const TraceParams &p, WaveParams w, WaveProgress &progress, cudaStream_t stream,
                             WaveRun *run, StageMarks *marks);
cudaError_t launch_closest_hit(const TraceParams &p, const sg_ray *rays, sg_hit *hits, uint32_t n,
                               cudaStream_t stream);
cudaError_t launch_light_visibility(const TraceParams &p, const sg_ray *rays, const uint32_t *lights,
                                    float *out, uint32_t n, cudaStream_t stream);
cudaError_t launch_ring_probe(const TraceParams &p, const sg_ray *rays, uint32_t body, float *out,
                              uint32_t n, cudaStream_t stream);
cudaError_t launch_terrain_probe(const TraceParams &p, const float *rays, float *out, uint32_t n,
                                 cudaStream_t stream);
// FMA-chain kernel of `blocks` x 256 threads, 128 * iters FMAs per thread.
cudaError_t launch_fma_peak(int blocks, int iters, float *out, cudaStream_t stream);
cudaError_t launch_ring_energy(float albedo, float tau, float mu, uint32_t steps, float *out,
                               cudaStream_t stream);

// ---------------------------------------------------------------------------
// Display (sg_display.cu): exposure metering and the HDR -> display resolve.
// ---------------------------------------------------------------------------
constexpr uint32_t kExposureBins = 256;

// The exposure state the reference shares with its shaders
// (pathtracer.rs:54-64): `value` is eased on the device by the metering.
struct ExposureState {
    float value, key, percentile, enabled, bias;
};

struct DisplayParams {
    const float4 *mean;      // width * height accumulation
    const float4 *backdrop;  // width * height Milky Way backdrop, or null
    uint32_t width, height;  // trace resolution
    uint32_t out_width, out_height;
    int format;              // SG_DISPLAY_RGBA8_SRGB or SG_DISPLAY_RGBA32F
    void *out;               // out_width * out_height pixels
    int automatic;           // use state->value instead of `manual`
    const ExposureState *state;
    float manual, bias, milky_way;
};

// Clears `histogram`, bins the central region of the accumulation and eases
// state->value towards the metered exposure (when state->enabled).
cudaError_t launch_exposure(const float4 *mean, uint32_t width, uint32_t height, uint32_t *histogram,
                            ExposureState *state, cudaStream_t stream);
cudaError_t launch_display(const DisplayParams &d, cudaStream_t stream);

// Flat parameter space of the adjoint's gradient buffer:
//   [0, kGradColor)          ring-table optical depths, slot * MAX_BINS + bin
//   [kGradColor, kGradMap)   per body: ring albedo rgb, then body colour rgb
//   [kGradMap, + texels)     albedo-map texels
constexpr uint32_t kGradColor = SG_RING_TABLE_SLOTS * SG_RING_TABLE_MAX_BINS;
constexpr uint32_t kGradMap = kGradColor + 6u * SG_BODY_CAPACITY;

// What an adjoint launch reads beyond the integrator's parameters.
struct AdjointParams {
    const float4 *dl_dimage;          // d loss / d accumulated pixel (w ignored)
    float inv_samples;                // 1 / samples behind the accumulation
    float *grad;                      // kGradMap + texels floats, accumulated
    uint32_t tau_window;              // shared-memory window over [0, tau_window)
    uint32_t color_window;            // ... and over [kGradColor, + color_window)
    unsigned long long *overflow;     // derivative entries dropped (full lists)
    // Vertex checkpoints of the forward (ck.totals null: replay every sample
    // from its seed). ck.sample_base: accumulation index of the launch's
    // first sample.
    Checkpoints ck;
};

// The segments between the forward's vertex checkpoints: one thread per
// stored record, `records` of them (sg_set_checkpoints).
cudaError_t launch_checkpoint_segments(const TraceParams &p, const AdjointParams &a, uint32_t records,
                                       cudaStream_t stream);

// Dynamic shared memory of an adjoint launch.
size_t adjoint_smem_bytes(const TraceParams &p, const AdjointParams &a);

// Replay the launch's samples (sampling.x, counts.z as for launch_trace)
// and accumulate the loss gradient into a.grad; the image is not touched.
cudaError_t launch_adjoint(const TraceParams &p, const AdjointParams &a, cudaStream_t stream);

// ---------------------------------------------------------------------------
// Staged adjoint (sg_wave_adjoint.cu): the same replay in the wavefront's
// extend / ring / surface stages. A path holds one adjoint slot (its
// persistent derivative state and lists) from its first surviving extend
// to its end; free slots circulate through a ring of slot ids.
// ---------------------------------------------------------------------------
constexpr uint32_t kAdjointSideVec4 = 10;  // float4 words of one slot's state

struct AdjointWave {
    float4 *side;         // kAdjointSideVec4 float4 per slot
    uint4 *queued;        // 2 * pool: per ring-queue entry, then per surface-queue entry,
                          // (slot, pixel, sample, 1 if the sample starts in this iteration)
    void *lists;          // one PrbLists per slot
    uint32_t *free_ring;  // `pool` slot ids: give-back k writes position k % pool
    uint32_t *free_ends;  // [0] allocations, [1] give-backs so far (monotonic)
};

// Bytes of the adjoint slots for `pool` paths.
size_t adjoint_slot_bytes(uint32_t pool);

// Makes every slot of `x` free (both counters to zero: allocation j < pool
// takes slot j); once per backward call.
cudaError_t reset_adjoint_slots(const AdjointWave &x, uint32_t pool, cudaStream_t stream);

// The samples of `p` (as launch_adjoint) through the stages; returns once
// they have drained (host checks as launch_wavefront).
cudaError_t launch_adjoint_wavefront(const TraceParams &p, const AdjointParams &a, WaveParams w,
                                     const AdjointWave &x, WaveProgress &progress, cudaStream_t stream, WaveRun *run);

}  // namespace sg
