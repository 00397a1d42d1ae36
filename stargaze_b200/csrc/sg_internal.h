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
};

constexpr int kEventCount = 9;

// Shared-memory bytes a launch with these parameters needs.
size_t trace_smem_bytes(const TraceParams &p);

cudaError_t launch_trace(const TraceParams &p, bool count_events, cudaStream_t stream);
cudaError_t launch_closest_hit(const TraceParams &p, const sg_ray *rays, sg_hit *hits, uint32_t n,
                               cudaStream_t stream);
cudaError_t launch_light_visibility(const TraceParams &p, const sg_ray *rays, const uint32_t *lights,
                                    float *out, uint32_t n, cudaStream_t stream);
cudaError_t launch_ring_probe(const TraceParams &p, const sg_ray *rays, uint32_t body, float *out,
                              uint32_t n, cudaStream_t stream);
// FMA-chain kernel of `blocks` x 256 threads, 128 * iters FMAs per thread.
cudaError_t launch_fma_peak(int blocks, int iters, float *out, cudaStream_t stream);
cudaError_t launch_ring_energy(float albedo, float tau, float mu, uint32_t steps, float *out,
                               cudaStream_t stream);

}  // namespace sg
