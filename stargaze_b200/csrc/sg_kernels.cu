// sg_kernels.cu — integrator and probe kernels for sm_100a.
//
// The integrator is a per-pixel megakernel: one thread owns one pixel, runs
// the dispatch's samples through trace() and folds the batch into a
// Kahan-compensated per-pixel sum. CTAs cover 16x16 pixel tiles and each
// warp an 8x4 sub-tile, so neighbouring lanes trace neighbouring pixels and
// take the same branches as long as possible.
#include <algorithm>

#include "sg_wave_common.cuh"

namespace sg {

namespace {

__device__ __forceinline__ void flush_events(const Events &ev, unsigned long long *events) {
    const uint32_t v[kEventCount] = {ev.vertices,      ev.sphere_tests,      ev.sphere_hits, ev.ring_tests,
                                     ev.light_samples, ev.shadow_rays,       ev.ring_events, ev.surface_events,
                                     ev.rng_draws,     ev.terrain_nodes,     ev.terrain_triangles,
                                     ev.prop_boxes,    ev.prop_tests};
#pragma unroll
    for (int k = 0; k < kEventCount; ++k) {
        unsigned long long x = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31u) == 0u && events) atomicAdd(&events[k], x);
    }
}

// Resident CTAs per SM the integrator is compiled for (register budget
// 65536 / (256 * SG_TRACE_MIN_BLOCKS) per thread). Measured on the ring
// workload: 1 CTA/SM 1846, 2 CTAs 2465, 3 CTAs 2882, 4 CTAs 2981 Msamples/s —
// more resident warps hide instruction-fetch and dependency latency better
// than the extra registers save spills.
#ifndef SG_TRACE_MIN_BLOCKS
#define SG_TRACE_MIN_BLOCKS 4
#endif

template <bool C, bool L, bool F, bool A>
__global__ void __launch_bounds__(kThreads, SG_TRACE_MIN_BLOCKS) trace_kernel(const __grid_constant__ TraceParams P) {
    extern __shared__ float4 smem[];
    const Scene S = stage_scene(P, smem);
    Events ev{};
    const Counter<C, L, F> K{&ev};
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t x = blockIdx.x * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t y = blockIdx.y * kTile + (warp >> 1) * 4u + (lane >> 3);
    if (x < P.width && y < P.height) {
        const uint32_t pixel = y * P.width + x;
        const uint32_t z = P.s.counts[2];
        // Lanes of a warp trace the same sample index in lockstep: adjacent
        // pixels then sit at the same vertex type (camera ray, ring event,
        // bounce) far more often than with per-lane path regeneration, which
        // measured 20 % slower on the ring workload.
        float4 total = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float3 sky = f3(0.0f, 0.0f, 0.0f);
        Path path;
        Forward<A> nograd;
        const Cull cull = camera_cull<C>(P, blockIdx.y * gridDim.x + blockIdx.x);
        for (uint32_t smp = 0; smp < z; ++smp) {
            start_path(path, &P.s, K, pixel, x, y, smp);
            // The camera ray takes the tile's cull masks, later rays none.
            if (!step(S, K, path, nograd, cull)) {
                while (!step(S, K, path, nograd)) {
                }
            }
            const float4 r = finish_path(path);
            total.x += r.x;
            total.y += r.y;
            total.z += r.z;
            total.w += r.w;
            sky = sky + path.backdrop;
        }
        if (P.sky_on) fold_backdrop(P, pixel, sky);
        // Progressive accumulation: the WGSL keeps a running mean
        // (pathtrace.wgsl:1662-1674); here the per-pixel sum is compensated
        // (Kahan) and the mean re-derived from it.
        const uint32_t old_count = P.s.counts[1];
        const float new_count = (float)(old_count + z);
        float4 sum, comp;
        if (old_count == 0u) {
            sum = total;
            comp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        } else {
            sum = P.sum[pixel];
            comp = P.comp[pixel];
            float yv, t;
            yv = __fsub_rn(total.x, comp.x); t = __fadd_rn(sum.x, yv); comp.x = __fsub_rn(__fsub_rn(t, sum.x), yv); sum.x = t;
            yv = __fsub_rn(total.y, comp.y); t = __fadd_rn(sum.y, yv); comp.y = __fsub_rn(__fsub_rn(t, sum.y), yv); sum.y = t;
            yv = __fsub_rn(total.z, comp.z); t = __fadd_rn(sum.z, yv); comp.z = __fsub_rn(__fsub_rn(t, sum.z), yv); sum.z = t;
            yv = __fsub_rn(total.w, comp.w); t = __fadd_rn(sum.w, yv); comp.w = __fsub_rn(__fsub_rn(t, sum.w), yv); sum.w = t;
        }
        P.sum[pixel] = sum;
        P.comp[pixel] = comp;
        P.mean[pixel] = make_float4(__fdiv_rn(__fsub_rn(sum.x, comp.x), new_count),
                                    __fdiv_rn(__fsub_rn(sum.y, comp.y), new_count),
                                    __fdiv_rn(__fsub_rn(sum.z, comp.z), new_count),
                                    __fdiv_rn(__fsub_rn(sum.w, comp.w), new_count));
    }
    if constexpr (C) flush_events(ev, P.events);
}

// ---------------------------------------------------------------------------
// Path-replay adjoint
// ---------------------------------------------------------------------------
// One sample's derivative: pass 1 replays the path without derivatives and
// records what pass 2 needs to weigh each factor by the radiance gathered
// after it (sg_adjoint.cuh); pass 2 replays it again and scatters.
// A path whose ring-indirect cap does not bind ends after pass 1 (its
// deferred factors flushed); the others replay once more. `lanes`: the
// warp's lanes that run the same samples; they meet after each pass so that
// a warp replays one pass at a time (lanes left to drift between the two
// passes would run two copies of the integrator apart).
// Replays a checkpointed path from `path` until a scatter brings its depth
// to `end_depth`, where the next segment's record starts, or it ends.
template <bool L, bool F>
__device__ __forceinline__ void replay_segment(const Scene &S, Counter<false, L, F> K, Prb &G, Path &path,
                                               uint32_t end_depth, Cull first = kTestAll) {
    if (step(S, K, path, G, first) || path.depth >= end_depth) return;
    while (!step(S, K, path, G)) {
        if (path.depth >= end_depth) break;
    }
}

template <bool L, bool F>
__device__ __forceinline__ void adjoint_sample(const Scene &S, Counter<false, L, F> K, Prb &G, float3 w, uint32_t pixel,
                                               uint32_t x, uint32_t y, uint32_t smp, unsigned lanes,
                                               uint32_t segment_end, Cull cull) {
    bool again = true;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        if (again) {
            Path path;
            start_path(path, S.s, K, pixel, x, y, smp);
            if (segment_end) {
                // A checkpointed sample: its first segment, once.
                replay_segment(S, K, G, path, segment_end, cull);
                again = false;
            } else {
                // The camera ray takes the tile's cull masks.
                if (!step(S, K, path, G, cull)) {
                    while (!step(S, K, path, G)) {
                    }
                }
                if (pass == 0) {
                    again = G.deferral_full || cap_binds(G, path.radiance);
                    if (again) pass2_setup(G, path.radiance, w);
                    else flush_deferred(G);
                }
            }
        }
        __syncwarp(lanes);
    }
}

// Resident CTAs per SM the adjoint is compiled for.
#ifndef SG_ADJOINT_MIN_BLOCKS
#define SG_ADJOINT_MIN_BLOCKS 2
#endif

template <bool L, bool F>
__global__ void __launch_bounds__(kThreads, SG_ADJOINT_MIN_BLOCKS)
    adjoint_kernel(const __grid_constant__ TraceParams P, const __grid_constant__ AdjointParams A) {
    extern __shared__ float4 smem[];
    // Dynamic shared memory: bodies and staged tables (stage_scene), the
    // inverse colours (2 float4 per body), then the gradient windows.
    const uint32_t n_bodies = P.s.counts[0];
    float4 *inv = smem + trace_smem_floats(P) / 4u;
    float *window = reinterpret_cast<float *>(inv + 2u * n_bodies);
    const uint32_t window_n = A.tau_window + A.color_window;
    for (uint32_t k = threadIdx.x; k < window_n; k += blockDim.x) window[k] = 0.0f;
    for (uint32_t k = threadIdx.x; k < n_bodies; k += blockDim.x) {
        const float4 m = P.bodies[k * kBodyVec4 + kMaterial], r = P.bodies[k * kBodyVec4 + kRingColor];
        inv[2u * k] = make_float4(inv_or_zero(m.x), inv_or_zero(m.y), inv_or_zero(m.z), 0.0f);
        inv[2u * k + 1u] = make_float4(inv_or_zero(r.x), inv_or_zero(r.y), inv_or_zero(r.z), 0.0f);
    }
    const Scene S = stage_scene(P, smem);  // synchronises the block
    const Counter<false, L, F> K{nullptr};
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t x = blockIdx.x * kTile + (warp & 1u) * 8u + (lane & 7u);
    const uint32_t y = blockIdx.y * kTile + (warp >> 1) * 4u + (lane >> 3);
    float own[6u * kColorSlots];
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) own[k] = 0.0f;
    const uint32_t own_n = 6u * (n_bodies < kColorSlots ? n_bodies : kColorSlots);
    PrbLists lists;
    float4 local[kMaxLocal];
    Prb G;
    G.lists = &lists;
    G.local = local;
    G.local_stride = 1u;
    G.sink = GradSink{own, own_n, window, A.tau_window, window + A.tau_window, A.color_window, A.grad, 1u};
    G.inv = inv;
    G.dropped = 0;
    const bool inside = x < P.width && y < P.height;
    const uint32_t pixel = inside ? y * P.width + x : 0u;
    float3 w = f3(0.0f, 0.0f, 0.0f);
    if (inside) {
        const float4 d = A.dl_dimage[pixel];
        w = f3(d.x, d.y, d.z) * A.inv_samples;
    }
    const bool busy = w.x != 0.0f || w.y != 0.0f || w.z != 0.0f;
    const unsigned lanes = __ballot_sync(0xffffffffu, busy);
    const Cull cull = camera_cull<false>(P, blockIdx.y * gridDim.x + blockIdx.x);
    if (busy) {
        const uint32_t z = P.s.counts[2];
        const uint32_t pixels = P.width * P.height;
#pragma unroll 1
        for (uint32_t smp = 0; smp < z; ++smp) {
            // With the forward's checkpoints, a sample that has them (and no
            // binding cap) replays only up to its first one; the segment
            // kernel replays the rest.
            uint32_t segment_end = 0;
            if (A.ck.totals && A.ck.sample_base + smp < A.ck.samples) {
                const float4 t = A.ck.totals[(size_t)(A.ck.sample_base + smp) * pixels + pixel];
                if ((__float_as_uint(t.w) & 3u) == 1u) {
                    segment_setup(G, w, f3(t.x, t.y, t.z), f3(0.0f, 0.0f, 0.0f));
                    segment_end = A.ck.every;
                }
            }
            if (!segment_end) pass1_setup(G, w);
            adjoint_sample(S, K, G, w, pixel, x, y, smp, lanes, segment_end, cull);
        }
    }
    // Per-thread colour sums: reduce over the warp, then into the window.
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) {
        float v = own[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0u && v != 0.0f) {
            if (k < A.color_window) atomicAdd(window + A.tau_window + k, v);
            else atomicAdd(A.grad + kGradColor + k, v);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < window_n; k += blockDim.x) {
        const float v = window[k];
        if (v != 0.0f) atomicAdd(A.grad + (k < A.tau_window ? k : kGradColor + (k - A.tau_window)), v);
    }
    unsigned long long dropped = G.dropped;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dropped += __shfl_down_sync(0xffffffffu, dropped, o);
    if (lane == 0u && dropped != 0ull && A.overflow) atomicAdd(A.overflow, dropped);
}

// The segments between vertex checkpoints: one thread per record of the
// forward (Checkpoints), replaying from the stored state with the weights of
// the path's known total until the next checkpoint depth or the path's end.
// Gradient sinks as in adjoint_kernel.
template <bool L, bool F>
__global__ void __launch_bounds__(kThreads, SG_ADJOINT_MIN_BLOCKS)
    segment_kernel(const __grid_constant__ TraceParams P, const __grid_constant__ AdjointParams A, uint32_t records) {
    extern __shared__ float4 smem[];
    const uint32_t n_bodies = P.s.counts[0];
    float4 *inv = smem + trace_smem_floats(P) / 4u;
    float *window = reinterpret_cast<float *>(inv + 2u * n_bodies);
    const uint32_t window_n = A.tau_window + A.color_window;
    for (uint32_t k = threadIdx.x; k < window_n; k += blockDim.x) window[k] = 0.0f;
    for (uint32_t k = threadIdx.x; k < n_bodies; k += blockDim.x) {
        const float4 m = P.bodies[k * kBodyVec4 + kMaterial], r = P.bodies[k * kBodyVec4 + kRingColor];
        inv[2u * k] = make_float4(inv_or_zero(m.x), inv_or_zero(m.y), inv_or_zero(m.z), 0.0f);
        inv[2u * k + 1u] = make_float4(inv_or_zero(r.x), inv_or_zero(r.y), inv_or_zero(r.z), 0.0f);
    }
    const Scene S = stage_scene(P, smem);  // synchronises the block
    const Counter<false, L, F> K{nullptr};
    const uint32_t lane = threadIdx.x & 31u;
    float own[6u * kColorSlots];
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) own[k] = 0.0f;
    const uint32_t own_n = 6u * (n_bodies < kColorSlots ? n_bodies : kColorSlots);
    PrbLists lists;
    float4 local[kMaxLocal];
    Prb G;
    G.lists = &lists;
    G.local = local;
    G.local_stride = 1u;
    G.sink = GradSink{own, own_n, window, A.tau_window, window + A.tau_window, A.color_window, A.grad, 1u};
    G.inv = inv;
    G.dropped = 0;
    const uint32_t pixels = P.width * P.height;
#pragma unroll 1
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < records; r += gridDim.x * blockDim.x) {
        Path path;
        const uint3 key = load_checkpoint(A.ck, r, path);  // (pixel, sample, depth)
        path.backdrop = f3(0.0f, 0.0f, 0.0f);
        path.sample = 0u;
        const float4 t = A.ck.totals[(size_t)key.y * pixels + key.x];
        if (__float_as_uint(t.w) & 2u) continue;  // replayed from its seed
        const float4 d = A.dl_dimage[key.x];
        const float3 w = f3(d.x, d.y, d.z) * A.inv_samples;
        if (w.x == 0.0f && w.y == 0.0f && w.z == 0.0f) continue;
        segment_setup(G, w, f3(t.x, t.y, t.z), path.radiance);
        const uint32_t next = key.z + A.ck.every;
        replay_segment(S, K, G, path, next <= A.ck.max_depth ? next : 0xffffffffu);
    }
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) {
        float v = own[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0u && v != 0.0f) {
            if (k < A.color_window) atomicAdd(window + A.tau_window + k, v);
            else atomicAdd(A.grad + kGradColor + k, v);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < window_n; k += blockDim.x) {
        const float v = window[k];
        if (v != 0.0f) atomicAdd(A.grad + (k < A.tau_window ? k : kGradColor + (k - A.tau_window)), v);
    }
    unsigned long long dropped = G.dropped;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dropped += __shfl_down_sync(0xffffffffu, dropped, o);
    if (lane == 0u && dropped != 0ull && A.overflow) atomicAdd(A.overflow, dropped);
}

__device__ __forceinline__ Ray load_ray(const sg_ray &in) {
    return Ray{f3(in.offset[0], in.offset[1], in.offset[2]), f3(in.direction[0], in.direction[1], in.direction[2]),
               in.anchor};
}

template <bool F>
__global__ void __launch_bounds__(kThreads) closest_hit_kernel(const __grid_constant__ TraceParams P,
                                                               const sg_ray *rays, sg_hit *hits, uint32_t n) {
    extern __shared__ float4 smem[];
    const Scene S = stage_scene(P, smem);
    const Counter<false, true, F> K{nullptr};
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const sg_ray in = rays[k];
    const Ray r = load_ray(in);
    // An anchor outside the body table would index past the staged bodies.
    const bool valid = in.anchor == kMiss || in.anchor < P.s.counts[0];
    const Hit h = valid ? closest_hit(S, K, r) : Hit{1.0e30f, kMiss, 0.0f, f3(0.0f, 0.0f, 0.0f)};
    sg_hit out;
    out.distance = h.t;
    out.index = h.index;
    float3 nrm = f3(0.0f, 0.0f, 0.0f);
    if (h.index != kMiss) nrm = h.index >= kLocalBase ? h.n : sphere_normal(S, r, h.index, h.delta);
    out.normal[0] = nrm.x;
    out.normal[1] = nrm.y;
    out.normal[2] = nrm.z;
    hits[k] = out;
}

template <bool F>
__global__ void __launch_bounds__(kThreads) visibility_kernel(const __grid_constant__ TraceParams P,
                                                              const sg_ray *rays, const uint32_t *lights,
                                                              float *out, uint32_t n) {
    extern __shared__ float4 smem[];
    const Scene S = stage_scene(P, smem);
    const Counter<false, true, F> K{nullptr};
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const sg_ray in = rays[k];
    const uint32_t light = lights[k];
    const bool valid = (in.anchor == kMiss || in.anchor < P.s.counts[0]) && light < P.s.counts[0];
    out[k] = valid ? light_visibility(S, K, load_ray(in), light) : 0.0f;
}

template <bool F>
__global__ void __launch_bounds__(kThreads) ring_probe_kernel(const __grid_constant__ TraceParams P,
                                                              const sg_ray *rays, uint32_t body, float *out,
                                                              uint32_t n) {
    extern __shared__ float4 smem[];
    const Scene S = stage_scene(P, smem);
    const Counter<false, true, F> K{nullptr};
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const sg_ray in = rays[k];
    const Ray r = load_ray(in);
    float4 result = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (body < P.s.counts[0] && (in.anchor == kMiss || in.anchor < P.s.counts[0])) {
        const RingHit h = ring_hit(S, K, r, body);
        if (h.index != kMiss)
            result = make_float4(h.t, __fdiv_rn(length_rn(h.p), b_radius(S, body)), ring_transmission(S, r, h), 1.0f);
    }
    // Scalar stores: a caller's device pointer need only be 4-byte aligned.
    out[4 * k + 0] = result.x;
    out[4 * k + 1] = result.y;
    out[4 * k + 2] = result.z;
    out[4 * k + 3] = result.w;
}

__global__ void __launch_bounds__(kThreads) terrain_probe_kernel(const __grid_constant__ TraceParams P,
                                                                 const float *rays, float *out, uint32_t n) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float4 result = make_float4(0.0f, 0.0f, 0.0f, 1.0e30f);
    if (P.terrain) {
        const float3 o = f3(rays[6 * k], rays[6 * k + 1], rays[6 * k + 2]);
        const float3 d = f3(rays[6 * k + 3], rays[6 * k + 4], rays[6 * k + 5]);
        result = terrain_query<false>(P.terrain, P.terrain_cells, P.s.g.ground_up[3],
                                      (P.s.g.ground_counts[2] & 255u) == 3u, o, d, 1.0e29f, false, nullptr);
    }
    out[4 * k + 0] = result.x;
    out[4 * k + 1] = result.y;
    out[4 * k + 2] = result.z;
    out[4 * k + 3] = result.w;
}

__global__ void ring_energy_kernel(float albedo, float tau, float mu, uint32_t steps, float *out) {
    // ring_tests.rs:365-377: unscattered transmission plus both scattered
    // hemispheres, midpoint rule in the incoming cosine.
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const Optics o{f3(albedo, albedo, albedo), tau};
    float energy = expf(-tau / mu);
    for (uint32_t i = 0; i < steps; ++i) {
        const float mi = ((float)i + 0.5f) / (float)steps;
        const float3 sum = ring_bsdf(o, mu, mi) + ring_bsdf(o, mu, -mi);
        energy += sum.x * (kTau * mi / (float)steps);
    }
    *out = energy;
}

// FMA-chain throughput kernel: eight independent chains per thread keep
// every FP32 pipe busy; the result is kept live by an impossible store.
__global__ void __launch_bounds__(256) fma_peak_kernel(float seed, int iters, float *out) {
    float a0 = seed + (float)threadIdx.x, a1 = a0 + 1.0f, a2 = a0 + 2.0f, a3 = a0 + 3.0f;
    float a4 = a0 + 4.0f, a5 = a0 + 5.0f, a6 = a0 + 6.0f, a7 = a0 + 7.0f;
    const float b = 0.999999f, c = 1.0e-7f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 1234.5678f) out[0] = s;
}

// cache_terrain_geometry (terrain.wgsl:242-285): node AABBs with curvature
// and a +-0.02 m margin, curved vertices and normals (12+12-bit packed on
// grids over 1024 cells). One thread per vertex; the first N threads also
// write one node each. Strict arithmetic keeps the cache bit-identical to an
// IEEE evaluation, so traversal decisions match the oracle.
__global__ void __launch_bounds__(256) terrain_cache_kernel(float *T, uint32_t cells, float r) {
    const uint32_t index = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t width = t_width(cells);
    const float scale = t_scale_r(r);
    if (index < t_nodes(cells)) {
        const uint3 node = t_node(index, cells);
        const float lo_x = t_coordinate(node.x, cells, scale), lo_z = t_coordinate(node.y, cells, scale);
        const float hi_x = t_coordinate(node.x + node.z, cells, scale), hi_z = t_coordinate(node.y + node.z, cells, scale);
        const float near_x = clampf(0.0f, lo_x, hi_x), near_z = clampf(0.0f, lo_z, hi_z);
        const float far_x = fmaxf(fabsf(lo_x), fabsf(hi_x)), far_z = fmaxf(fabsf(lo_z), fabsf(hi_z));
        const float lower = __fsub_rn(__fadd_rn(__fmul_rn(T[t_bounds(cells) + index * 2u], scale),
                                                t_curvature(far_x, far_z, r)), 0.02f);
        const float upper = __fadd_rn(__fadd_rn(__fmul_rn(T[t_bounds(cells) + index * 2u + 1u], scale),
                                                t_curvature(near_x, near_z, r)), 0.02f);
        float *c = T + t_cache(cells) + (size_t)index * 6u;
        c[0] = lo_x;
        c[1] = lower;
        c[2] = lo_z;
        c[3] = hi_x;
        c[4] = upper;
        c[5] = hi_z;
    }
    if (index >= t_vertices(cells)) return;
    const uint32_t x = index % width, z = index / width;
    const float px = t_coordinate(x, cells, scale), pz = t_coordinate(z, cells, scale);
    const float vy = __fadd_rn(__fmul_rn(T[z * width + x], scale), t_curvature(px, pz, r));
    const float denom =
        __fsqrt_rn(fmaxf(__fsub_rn(__fmul_rn(r, r), __fadd_rn(__fmul_rn(px, px), __fmul_rn(pz, pz))), 1.0f));
    const float gx = __fdiv_rn(px, denom), gz = __fdiv_rn(pz, denom);
    float3 normal;
    if (t_compact(cells)) {
        const uint32_t lox = x > 0u ? x - 1u : 0u, loz = z > 0u ? z - 1u : 0u;
        const uint32_t hix = x + 1u < cells ? x + 1u : cells, hiz = z + 1u < cells ? z + 1u : cells;
        const float dx = __fdiv_rn(__fsub_rn(T[z * width + hix], T[z * width + lox]),
                                   __fdiv_rn(__fsub_rn(t_coordinate(hix, cells, scale), t_coordinate(lox, cells, scale)), scale));
        const float dz = __fdiv_rn(__fsub_rn(T[hiz * width + x], T[loz * width + x]),
                                   __fdiv_rn(__fsub_rn(t_coordinate(hiz, cells, scale), t_coordinate(loz, cells, scale)), scale));
        normal = f3(__fadd_rn(-dx, gx), 1.0f, __fadd_rn(-dz, gz));
    } else {
        const uint32_t vertices = t_vertices(cells);
        normal = f3(__fadd_rn(-T[vertices + index], gx), 1.0f, __fadd_rn(-T[2u * vertices + index], gz));
    }
    normal = mul_rn(normal, __fdiv_rn(1.0f, length_rn(normal)));
    float *v = T + t_vertex_cache(cells) + (size_t)index * t_vertex_stride(cells);
    if (t_compact(cells)) {
        v[0] = vy;
        // WGSL round() is round-half-to-even, as rintf.
        const float ux = rintf(__fmul_rn(clampf(__fadd_rn(__fmul_rn(normal.x, 0.5f), 0.5f), 0.0f, 1.0f), 4095.0f));
        const float uz = rintf(__fmul_rn(clampf(__fadd_rn(__fmul_rn(normal.z, 0.5f), 0.5f), 0.0f, 1.0f), 4095.0f));
        v[1] = (float)((uint32_t)ux | ((uint32_t)uz << 12));
    } else {
        v[0] = px;
        v[1] = vy;
        v[2] = pz;
        v[3] = normal.x;
        v[4] = normal.y;
        v[5] = normal.z;
    }
}

}  // namespace

size_t terrain_source_floats(uint32_t cells) { return (size_t)t_source(cells); }
size_t terrain_floats(uint32_t cells) {
    return (size_t)t_vertex_cache(cells) + (size_t)t_vertices(cells) * t_vertex_stride(cells);
}

cudaError_t launch_terrain_cache(float *terrain, uint32_t cells, float radius_m, cudaStream_t stream) {
    const uint32_t threads = t_vertices(cells) > t_nodes(cells) ? t_vertices(cells) : t_nodes(cells);
    terrain_cache_kernel<<<(threads + 255u) / 256u, 256, 0, stream>>>(terrain, cells, radius_m);
    return cudaGetLastError();
}

cudaError_t launch_fma_peak(int blocks, int iters, float *out, cudaStream_t stream) {
    fma_peak_kernel<<<blocks, 256, 0, stream>>>(1.0f, iters, out);
    return cudaGetLastError();
}

// cache_surface_sky (terrain.wgsl:286-302): texel (x, y) holds the air's
// in-scatter along the local direction at azimuth 2 pi (x + 0.5) / 16 and
// elevation sine (y + 0.5) / 8, seen from the camera, with the random state
// the reference seeds per texel. Zero without terrain. Built with the
// settings of an accumulation's first dispatch (counts.y = 0).
template <bool F>
__global__ void __launch_bounds__(kThreads) sky_cache_kernel(const __grid_constant__ TraceParams P, float4 *out) {
    extern __shared__ float4 smem[];
    const Scene S = stage_scene(P, smem);
    const uint32_t index = threadIdx.x;
    if (index >= kSkyTexels) return;
    float3 light = f3(0.0f, 0.0f, 0.0f);
    if (P.s.g.atmo_params[3] > 0.5f && P.s.g.ground_counts[1] != 0u) {
        const uint32_t x = index % 16u, y = index / 16u;
        const float mu = ((float)y + 0.5f) / 8.0f;
        const float phi = kTau * ((float)x + 0.5f) / 16.0f;
        const float r = sqrtf(1.0f - mu * mu);
        const float3 dir = from_ground(S, f3(r * cosf(phi), mu, r * sinf(phi)));
        const Counter<false, true, F> K{nullptr};
        light = atmosphere(S, K, f3(0.0f, 0.0f, 0.0f), dir, 1.0e30f, hash_u32(index ^ 0x91ce452du), 0u).inscatter;
    }
    out[index] = make_float4(light.x, light.y, light.z, 0.0f);
}

size_t trace_smem_bytes(const TraceParams &p) {
    return (size_t)p.s.counts[0] * kBodyVec4 * sizeof(float4) + (size_t)p.staged_table_floats * sizeof(float);
}

static cudaError_t set_smem(const void *fn, size_t bytes) {
    if (bytes <= 48u * 1024u) return cudaSuccess;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Launch one instantiation of a kernel with `smem` bytes of dynamic shared
// memory and 256-thread CTAs.
template <typename... K, typename... A>
static cudaError_t launch_variant(void (*kernel)(K...), dim3 grid, size_t smem, cudaStream_t stream, A &&...args) {
    cudaError_t e = set_smem((const void *)kernel, smem);
    if (e != cudaSuccess) return e;
    kernel<<<grid, kThreads, smem, stream>>>(args...);
    return cudaGetLastError();
}

cudaError_t launch_trace(const TraceParams &p, bool count_events, cudaStream_t stream) {
    const size_t smem = trace_smem_bytes(p);
    const dim3 grid((p.width + kTile - 1) / kTile, (p.height + kTile - 1) / kTile);
    // The landscape instantiation only for frames that enable it: the
    // celestial one carries neither its registers nor its code.
    // Frames with host air or styled bodies run the instantiations that
    // carry that code; the event-counting ones always do (gated at run time
    // there).
    const bool land = p.s.g.ground_north[3] != 0.0f;
    const int which =
        (count_events ? 8 : 0) | (p.air_on || p.styled ? 4 : 0) | (land ? 2 : 0) | (p.fp64_sites ? 1 : 0);
    switch (which) {
        case 0: return launch_variant(trace_kernel<false, false, false, false>, grid, smem, stream, p);
        case 1: return launch_variant(trace_kernel<false, false, true, false>, grid, smem, stream, p);
        case 2: return launch_variant(trace_kernel<false, true, false, false>, grid, smem, stream, p);
        case 3: return launch_variant(trace_kernel<false, true, true, false>, grid, smem, stream, p);
        case 4: return launch_variant(trace_kernel<false, false, false, true>, grid, smem, stream, p);
        case 5: return launch_variant(trace_kernel<false, false, true, true>, grid, smem, stream, p);
        case 6: return launch_variant(trace_kernel<false, true, false, true>, grid, smem, stream, p);
        case 7: return launch_variant(trace_kernel<false, true, true, true>, grid, smem, stream, p);
        case 8: case 12: return launch_variant(trace_kernel<true, false, false, true>, grid, smem, stream, p);
        case 9: case 13: return launch_variant(trace_kernel<true, false, true, true>, grid, smem, stream, p);
        case 10: case 14: return launch_variant(trace_kernel<true, true, false, true>, grid, smem, stream, p);
        default: return launch_variant(trace_kernel<true, true, true, true>, grid, smem, stream, p);
    }
}

cudaError_t launch_sky_cache(const TraceParams &p, float4 *out, cudaStream_t stream) {
    const size_t smem = trace_smem_bytes(p);
    if (p.fp64_sites) return launch_variant(sky_cache_kernel<true>, dim3(1), smem, stream, p, out);
    return launch_variant(sky_cache_kernel<false>, dim3(1), smem, stream, p, out);
}

size_t adjoint_smem_bytes(const TraceParams &p, const AdjointParams &a) {
    return trace_smem_bytes(p) + (size_t)p.s.counts[0] * 2u * sizeof(float4) +
           (size_t)(a.tau_window + a.color_window) * sizeof(float);
}

cudaError_t launch_adjoint(const TraceParams &p, const AdjointParams &a, cudaStream_t stream) {
    const size_t smem = adjoint_smem_bytes(p, a);
    const dim3 grid((p.width + kTile - 1) / kTile, (p.height + kTile - 1) / kTile);
    const bool land = p.s.g.ground_north[3] != 0.0f;
    switch ((land ? 2 : 0) | (p.fp64_sites ? 1 : 0)) {
        case 0: return launch_variant(adjoint_kernel<false, false>, grid, smem, stream, p, a);
        case 1: return launch_variant(adjoint_kernel<false, true>, grid, smem, stream, p, a);
        case 2: return launch_variant(adjoint_kernel<true, false>, grid, smem, stream, p, a);
        default: return launch_variant(adjoint_kernel<true, true>, grid, smem, stream, p, a);
    }
}

// Whether a sphere of radius `rho` at `c` (telescope space, camera at the
// origin) can meet a ray inside the cone of half-angle `alpha` about the
// unit direction `axis`: the directions that hit an external sphere form
// the cone of half-angle asin(rho / |c|) about c. Radius and angles carry
// margins (1e-3 relative, 1e-3 rad) far above the f32 error of the exact
// intersection tests, so a false here is a certain miss there.
__device__ __forceinline__ bool cone_meets_sphere(double3 axis, double alpha, double3 c, double rho) {
    const double dist = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
    const double r = rho * (1.0 + 1.0e-3);
    if (!(dist > r)) return true;  // the camera is inside or at the sphere (or the input is not finite)
    const double cosb = fmin(fmax((axis.x * c.x + axis.y * c.y + axis.z * c.z) / dist, -1.0), 1.0);
    return acos(cosb) <= alpha + asin(r / dist) + 1.0e-3;
}

__device__ __forceinline__ double3 unit_direction(double ndc_x, double ndc_y, double tangent, double aspect) {
    const double x = ndc_x * tangent * aspect, y = ndc_y * tangent;
    const double inv = 1.0 / sqrt(x * x + y * y + 1.0);
    return make_double3(x * inv, y * inv, -inv);
}

// One CTA per 16x16 tile, one thread per body: the bodies (their point
// discs included) and the rings a camera ray of the tile may meet. A camera
// ray of pixel (x, y) has ndc in [2x/W - 1, 2(x+1)/W - 1] x [1 - 2(y+1)/H,
// 1 - 2y/H] (camera_direction, pathtrace.wgsl:1619-1626); the tile's rays
// lie in the cone about its centre ray through its farthest corner.
__global__ void __launch_bounds__(32) camera_cull_kernel(const __grid_constant__ TraceParams P, uint2 *out,
                                                         uint32_t tiles_x) {
    const uint32_t tx = blockIdx.x % tiles_x, ty = blockIdx.x / tiles_x;
    const uint32_t i = threadIdx.x;
    const uint32_t n = P.s.counts[0];
    bool body = false, ring = false;
    if (i < n) {
        const double w = P.s.g.viewport[0], h = P.s.g.viewport[1];
        const double tangent = P.s.g.cam_forward[3], aspect = P.s.g.viewport[3];
        const double x0 = 2.0 * (tx * kTile) / w - 1.0, x1 = 2.0 * fmin((double)(tx * kTile + kTile), w) / w - 1.0;
        const double y0 = 1.0 - 2.0 * fmin((double)(ty * kTile + kTile), h) / h, y1 = 1.0 - 2.0 * (ty * kTile) / h;
        const double3 axis = unit_direction(0.5 * (x0 + x1), 0.5 * (y0 + y1), tangent, aspect);
        double alpha = 0.0;
        const double cx[2] = {x0, x1}, cy[2] = {y0, y1};
        for (int a = 0; a < 2; ++a)
            for (int b = 0; b < 2; ++b) {
                const double3 d = unit_direction(cx[a], cy[b], tangent, aspect);
                const double c = fmin(fmax(d.x * axis.x + d.y * axis.y + d.z * axis.z, -1.0), 1.0);
                alpha = fmax(alpha, acos(c));
            }
        const float4 hi = P.bodies[i * kBodyVec4 + kCenter], lo = P.bodies[i * kBodyVec4 + kLow];
        const double3 c = make_double3((double)hi.x + lo.x, (double)hi.y + lo.y, (double)hi.z + lo.z);
        const double dist = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
        // point_disc_hit draws an unresolved body as a disc of at least
        // `angle` radians (pathtrace.wgsl:1308-1333).
        const double pixel = 2.0 * tangent / fmax(h, 1.0);
        const double angle = fmin(fmax((double)kPointDiscRadius, 0.7 * pixel), (double)kStarDotPixels * pixel);
        const double radius = hi.w;
        body = cone_meets_sphere(axis, alpha, c, fmax(radius, angle * dist));
        const float4 plane = P.bodies[i * kBodyVec4 + kRingPlane], params = P.bodies[i * kBodyVec4 + kRingParams];
        // The annulus lies inside the sphere of its outer radius.
        if (params.x > plane.w && params.y > 0.0f) ring = cone_meets_sphere(axis, alpha, c, (double)params.x * radius);
    }
    const uint32_t bodies = __ballot_sync(0xffffffffu, body), rings = __ballot_sync(0xffffffffu, ring);
    if (i == 0) out[blockIdx.x] = make_uint2(bodies, rings);
}

cudaError_t launch_camera_cull(const TraceParams &p, uint2 *out, cudaStream_t stream) {
    const uint32_t tiles_x = (p.width + kTile - 1) / kTile, tiles_y = (p.height + kTile - 1) / kTile;
    if (p.s.counts[0] > 32u || tiles_x * tiles_y == 0) return cudaErrorInvalidValue;
    camera_cull_kernel<<<tiles_x * tiles_y, 32, 0, stream>>>(p, out, tiles_x);
    return cudaGetLastError();
}

cudaError_t launch_checkpoint_segments(const TraceParams &p, const AdjointParams &a, uint32_t records,
                                       cudaStream_t stream) {
    if (records == 0) return cudaSuccess;
    const size_t smem = adjoint_smem_bytes(p, a);
    const bool land = p.s.g.ground_north[3] != 0.0f;
    const void *fn;
    switch ((land ? 2 : 0) | (p.fp64_sites ? 1 : 0)) {
        case 0: fn = (const void *)segment_kernel<false, false>; break;
        case 1: fn = (const void *)segment_kernel<false, true>; break;
        case 2: fn = (const void *)segment_kernel<true, false>; break;
        default: fn = (const void *)segment_kernel<true, true>; break;
    }
    int grid = 0;
    cudaError_t e = set_smem(fn, smem);
    if (e == cudaSuccess) e = persistent_grid(fn, smem, &grid);
    if (e != cudaSuccess) return e;
    grid = (int)std::min<uint32_t>((uint32_t)grid, (records + kThreads - 1) / kThreads);
    switch ((land ? 2 : 0) | (p.fp64_sites ? 1 : 0)) {
        case 0: segment_kernel<false, false><<<grid, kThreads, smem, stream>>>(p, a, records); break;
        case 1: segment_kernel<false, true><<<grid, kThreads, smem, stream>>>(p, a, records); break;
        case 2: segment_kernel<true, false><<<grid, kThreads, smem, stream>>>(p, a, records); break;
        default: segment_kernel<true, true><<<grid, kThreads, smem, stream>>>(p, a, records); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_closest_hit(const TraceParams &p, const sg_ray *rays, sg_hit *hits, uint32_t n,
                               cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t smem = trace_smem_bytes(p);
    const dim3 grid((n + kThreads - 1) / kThreads);
    if (p.fp64_sites) return launch_variant(closest_hit_kernel<true>, grid, smem, stream, p, rays, hits, n);
    return launch_variant(closest_hit_kernel<false>, grid, smem, stream, p, rays, hits, n);
}

cudaError_t launch_light_visibility(const TraceParams &p, const sg_ray *rays, const uint32_t *lights,
                                    float *out, uint32_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t smem = trace_smem_bytes(p);
    const dim3 grid((n + kThreads - 1) / kThreads);
    if (p.fp64_sites) return launch_variant(visibility_kernel<true>, grid, smem, stream, p, rays, lights, out, n);
    return launch_variant(visibility_kernel<false>, grid, smem, stream, p, rays, lights, out, n);
}

cudaError_t launch_ring_probe(const TraceParams &p, const sg_ray *rays, uint32_t body, float *out,
                              uint32_t n, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    const size_t smem = trace_smem_bytes(p);
    const dim3 grid((n + kThreads - 1) / kThreads);
    if (p.fp64_sites) return launch_variant(ring_probe_kernel<true>, grid, smem, stream, p, rays, body, out, n);
    return launch_variant(ring_probe_kernel<false>, grid, smem, stream, p, rays, body, out, n);
}

cudaError_t launch_terrain_probe(const TraceParams &p, const float *rays, float *out, uint32_t n,
                                 cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    terrain_probe_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, stream>>>(p, rays, out, n);
    return cudaGetLastError();
}

cudaError_t launch_ring_energy(float albedo, float tau, float mu, uint32_t steps, float *out,
                               cudaStream_t stream) {
    ring_energy_kernel<<<1, 32, 0, stream>>>(albedo, tau, mu, steps, out);
    return cudaGetLastError();
}

}  // namespace sg
