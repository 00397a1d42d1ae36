// sg_internal.h — launch interface between the C-ABI host runtime and the
// CUDA kernels of the integrator.
#pragma once

#include <cstdint>
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
    const float4 *props;
    const float4 *prop_trig;  // 2 float4 per prop: (sin, cos) of x, y; z
    uint32_t n_props;
    const float *albedo_map;
    uint32_t map_width, map_height;
    float map_extent;
    uint32_t fp64_sites;  // ring plane, host sphere and 5 mm offset in FP64
};

// Geometry cache of the heightfield (cache_terrain_geometry,
// terrain.wgsl:242-285) for host radius `radius_m`, in place.
cudaError_t launch_terrain_cache(float *terrain, uint32_t cells, float radius_m, cudaStream_t stream);

// Floats of the full device terrain layout for `cells` cells per side.
size_t terrain_floats(uint32_t cells);
size_t terrain_source_floats(uint32_t cells);

constexpr int kEventCount = 9;

// Shared-memory bytes a launch with these parameters needs.
size_t trace_smem_bytes(const TraceParams &p);

// Sets the message sg_last_error(NULL) returns (entry points without a
// context report through it).
void set_library_error(const char *message);

cudaError_t launch_trace(const TraceParams &p, bool count_events, cudaStream_t stream);
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
};

// Dynamic shared memory of an adjoint launch.
size_t adjoint_smem_bytes(const TraceParams &p, const AdjointParams &a);

// Replay the launch's samples (sampling.x, counts.z as for launch_trace)
// and accumulate the loss gradient into a.grad; the image is not touched.
cudaError_t launch_adjoint(const TraceParams &p, const AdjointParams &a, cudaStream_t stream);

}  // namespace sg
