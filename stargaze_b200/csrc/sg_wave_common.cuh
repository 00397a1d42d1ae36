// sg_wave_common.cuh — what the wavefront integrator and the staged adjoint
// share: the path state planes in HBM, CTA-aggregated queue appends, the
// per-iteration counters and the host helpers of the stage loop.
#pragma once

#include <vector>

#include "sg_integrator.cuh"

namespace sg {

namespace {

// Resident CTAs per SM the forward stages are compiled for (65536 / (256 x
// this) registers per thread).
#ifndef SG_WAVE_MIN_BLOCKS
#define SG_WAVE_MIN_BLOCKS 4
#endif
#ifndef SG_WAVE_EXTEND_MIN_BLOCKS
#define SG_WAVE_EXTEND_MIN_BLOCKS SG_WAVE_MIN_BLOCKS
#endif
#ifndef SG_WAVE_SHADE_MIN_BLOCKS
#define SG_WAVE_SHADE_MIN_BLOCKS SG_WAVE_MIN_BLOCKS
#endif
// Paths a thread of the extend stage takes per queue append (celestial
// frames). Measured on the 1080p ring step: 1 59.5 ms, 4 55.9, 6 55.1,
// 8 55.5.
#ifndef SG_WAVE_EXTEND_ITEMS
#define SG_WAVE_EXTEND_ITEMS 6
#endif

// ---------------------------------------------------------------------------
// Path state planes
// ---------------------------------------------------------------------------
//   0  ray.o, ray.anchor            4  ring_base, shine_body
//   1  ray.d, rng                   5  previous_vertex.o, previous_vertex.anchor
//   2  throughput, previous_pdf     6  iterations | point_gained << 31,
//   3  radiance, ring_cap              depth | null_crossings << 16 | in_air << 30
//                                      | sky_on_escape << 31, result slot,
//                                      checkpoint bits
// The previous vertex is only ever used for its position (relative_center),
// so its direction is not stored.
__device__ __forceinline__ float4 pack3(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float4 pack3u(float3 v, uint32_t w) { return make_float4(v.x, v.y, v.z, __uint_as_float(w)); }
__device__ __forceinline__ float3 xyz4(float4 v) { return f3(v.x, v.y, v.z); }

// Plane 6's first two words.
__device__ __forceinline__ float iteration_word(const Path &p) {
    return __uint_as_float(p.iterations | (p.point_gained ? 0x80000000u : 0u));
}
__device__ __forceinline__ float depth_word(const Path &p) {
    return __uint_as_float(p.depth | (p.null_crossings << 16) | (p.in_air ? 0x40000000u : 0u) |
                           (p.sky_on_escape ? 0x80000000u : 0u));
}

__device__ __forceinline__ void store_path(float4 *st, uint32_t pool, uint32_t i, const Path &p, uint32_t slot) {
    st[0 * pool + i] = pack3u(p.ray.o, p.ray.anchor);
    st[1 * pool + i] = pack3u(p.ray.d, p.rng);
    st[2 * pool + i] = pack3(p.throughput, p.previous_pdf);
    st[3 * pool + i] = pack3(p.radiance, p.ring_cap);
    st[4 * pool + i] = pack3u(p.ring_base, p.shine_body);
    st[5 * pool + i] = pack3u(p.previous_vertex.o, p.previous_vertex.anchor);
    st[6 * pool + i] = make_float4(iteration_word(p), depth_word(p), __uint_as_float(slot), __uint_as_float(p.ckpt));
}

// Planes 0, 1 and 6: what extend reads. Returns the result slot.
__device__ __forceinline__ uint32_t load_ray_part(const float4 *st, uint32_t pool, uint32_t i, Path &p) {
    const float4 a = st[0 * pool + i], b = st[1 * pool + i], g = st[6 * pool + i];
    p.ray = Ray{xyz4(a), xyz4(b), __float_as_uint(a.w)};
    p.rng = __float_as_uint(b.w);
    const uint32_t it = __float_as_uint(g.x), dn = __float_as_uint(g.y);
    p.iterations = it & 0x7fffffffu;
    p.point_gained = (it >> 31) != 0u;
    p.depth = dn & 0xffffu;
    p.null_crossings = (dn >> 16) & 0x3fffu;
    p.in_air = (dn & 0x40000000u) != 0u;
    p.sky_on_escape = (dn & 0x80000000u) != 0u;
    p.backdrop = f3(0.0f, 0.0f, 0.0f);  // set only where a path escapes, which ends it
    p.ckpt = __float_as_uint(g.w);
    return __float_as_uint(g.z);
}

// Planes 3 and 4: radiance and the ring cap (what finish_path reads) and
// the ringshine body.
__device__ __forceinline__ void load_radiance_part(const float4 *st, uint32_t pool, uint32_t i, Path &p) {
    const float4 c = st[3 * pool + i], d = st[4 * pool + i];
    p.radiance = xyz4(c);
    p.ring_cap = c.w;
    p.ring_base = xyz4(d);
    p.shine_body = __float_as_uint(d.w);
}

// Planes 2 and 5: the rest of the state the shade stages need.
__device__ __forceinline__ void load_shade_part(const float4 *st, uint32_t pool, uint32_t i, Path &p) {
    const float4 c = st[2 * pool + i], e = st[5 * pool + i];
    p.throughput = xyz4(c);
    p.previous_pdf = c.w;
    p.previous_vertex = Ray{xyz4(e), f3(0.0f, 0.0f, 0.0f), __float_as_uint(e.w)};
}

// ---------------------------------------------------------------------------
// Vertex checkpoints (Checkpoints in sg_internal.h)
// ---------------------------------------------------------------------------
// The ring-indirect cap clamps this finished path (as finish_path does).
__device__ __forceinline__ bool cap_clamps(const Path &p) {
    return p.ring_cap < 1.0e29f && luminance(p.radiance - p.ring_base) > p.ring_cap;
}

// Accumulation index of the chunk sample behind result slot `slot`.
__device__ __forceinline__ uint32_t checkpoint_sample(const Checkpoints &ck, uint32_t chunk_first, uint32_t pixels,
                                                      uint32_t slot) {
    return ck.sample_base + chunk_first + slot / pixels;
}

// A path's end: its radiance before the cap and its checkpoint bits.
__device__ __forceinline__ void checkpoint_total(const Checkpoints &ck, uint32_t chunk_first, uint32_t pixels,
                                                 uint32_t slot, const Path &p) {
    const uint32_t sample = checkpoint_sample(ck, chunk_first, pixels, slot);
    if (sample >= ck.samples) return;
    ck.totals[(size_t)sample * pixels + slot % pixels] = pack3u(p.radiance, p.ckpt | (cap_clamps(p) ? 2u : 0u));
}

// Record `r`: the path's state as the pool stores it, then its key.
__device__ __forceinline__ void store_checkpoint(const Checkpoints &ck, uint32_t r, const Path &p, uint32_t pixel,
                                                 uint32_t sample) {
    float4 *rec = ck.records + (size_t)r * kCheckpointVec4;
    store_path(rec, 1u, 0u, p, 0u);
    rec[kWavePlanes] = make_float4(__uint_as_float(pixel), __uint_as_float(sample), __uint_as_float(p.depth), 0.0f);
}

// Loads record `r` into a path; returns its key (pixel, sample, depth).
__device__ __forceinline__ uint3 load_checkpoint(const Checkpoints &ck, uint32_t r, Path &p) {
    const float4 *rec = ck.records + (size_t)r * kCheckpointVec4;
    load_ray_part(rec, 1u, 0u, p);
    load_radiance_part(rec, 1u, 0u, p);
    load_shade_part(rec, 1u, 0u, p);
    const float4 key = rec[kWavePlanes];
    return make_uint3(__float_as_uint(key.x), __float_as_uint(key.y), __float_as_uint(key.z));
}

// ---------------------------------------------------------------------------
// CTA-aggregated queue appends
// ---------------------------------------------------------------------------
// Each thread of the CTA passes `flag[q]` for Q queues; the thread gets its
// slot in each queue where its flag is set. One atomicAdd per queue and
// CTA; every thread of the CTA must call it. Consecutive calls alternate
// between two scratch blocks, so a call never overwrites counts that a
// slower warp of the previous call has yet to read. (One atomic per warp
// without the barriers measured slower: 4 % on the ring workload's forward,
// 30 % on the terrain's, 30 % on the ring adjoint — same-address atomics
// from every warp serialise in L2.)
template <int Q, int B = kThreads>
struct Append {
    uint32_t warp_counts[Q][B / 32];
    uint32_t base[Q];
};

template <int Q, int B = kThreads>
__device__ __forceinline__ void block_append(Append<Q, B> &sm, const bool (&flag)[Q], uint32_t *const (&counter)[Q],
                                             uint32_t (&slot)[Q]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t ballot[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        ballot[q] = __ballot_sync(0xffffffffu, flag[q]);
        if (lane == 0) sm.warp_counts[q][warp] = __popc(ballot[q]);
    }
    __syncthreads();
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        uint32_t total = 0;
        for (uint32_t w = 0; w < (uint32_t)B / 32u; ++w) {
            const uint32_t c = sm.warp_counts[q][w];
            sm.warp_counts[q][w] = total;  // exclusive prefix
            total += c;
        }
        sm.base[q] = total ? atomicAdd(counter[q], total) : 0u;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) slot[q] = sm.base[q] + sm.warp_counts[q][warp] + __popc(ballot[q] & below);
}

// The same for K items per thread: bit k of flags[q] marks the thread's
// item k for queue q. Slots follow item order first, then thread order, so
// a round's queue entries keep the order of its input (k * B + thread).
// One barrier pair per K items: warps whose items took longer wait once
// per round instead of once per item.
template <int Q, int K, int B = kThreads>
struct AppendK {
    uint32_t warp_counts[Q][K][B / 32];
    uint32_t base[Q];
};

template <int Q, int K, int B = kThreads>
__device__ __forceinline__ void block_append_k(AppendK<Q, K, B> &sm, const uint32_t (&flags)[Q],
                                               uint32_t *const (&counter)[Q], uint32_t (&slot)[Q][K]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t below = (1u << lane) - 1u;
    uint32_t ballot[Q][K];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            ballot[q][k] = __ballot_sync(0xffffffffu, (flags[q] >> k) & 1u);
            if (lane == 0) sm.warp_counts[q][k][warp] = __popc(ballot[q][k]);
        }
    }
    __syncthreads();
    if (threadIdx.x < Q) {
        const int q = threadIdx.x;
        uint32_t total = 0;
        for (int k = 0; k < K; ++k) {
            for (uint32_t w = 0; w < (uint32_t)B / 32u; ++w) {
                const uint32_t c = sm.warp_counts[q][k][w];
                sm.warp_counts[q][k][w] = total;  // exclusive prefix in (item, warp) order
                total += c;
            }
        }
        sm.base[q] = total ? atomicAdd(counter[q], total) : 0u;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
#pragma unroll
        for (int k = 0; k < K; ++k)
            slot[q][k] = sm.base[q] + sm.warp_counts[q][k][warp] + __popc(ballot[q][k] & below);
    }
}

__device__ __forceinline__ WaveCounters *counters(const WaveParams &W, uint32_t t) {
    return W.counters + (t % kWaveCounterSets);
}

// Samples of a chunk are numbered sample-major over the padded tile grid.
__device__ __forceinline__ uint32_t padded_pixels(const WaveParams &W) { return W.tiles_x * W.tiles_y * 256u; }

// Grid of a persistent stage kernel: every resident CTA slot of every SM.
// (Asking for the largest L1 share through the shared-memory carveout
// halved the forward's speed and did not help the adjoint: the driver's
// choice stays.)
inline cudaError_t persistent_grid(const void *fn, size_t smem, int *grid, int threads = kThreads) {
    int device = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    if (e != cudaSuccess) return e;
    *grid = sms * (per_sm > 0 ? per_sm : 1);
    return cudaSuccess;
}

// Iterations the host enqueues beyond the one whose start it inspects.
constexpr uint64_t kLookahead = 2;

// Records the end of iteration t.
inline cudaError_t iteration_done(WaveProgress &pr, uint64_t t, cudaStream_t stream) {
    return cudaEventRecord(pr.done[t % kProgressSlots], stream);
}

// What iteration s started from: the paths kept and the next sample.
struct WaveStart {
    uint32_t kept, next;
};
inline cudaError_t started(const WaveProgress &pr, uint64_t s, WaveStart *out) {
    cudaError_t e = cudaEventSynchronize(pr.done[s % kProgressSlots]);
    if (e != cudaSuccess) return e;
    const volatile uint2 *h = pr.host + s % kProgressSlots;
    out->kept = h->x;
    out->next = h->y;
    return cudaSuccess;
}

// Whether iteration s started with no path kept and no sample left (of
// `samples`): then it and every later iteration had nothing to do.
inline cudaError_t drained(const WaveProgress &pr, uint64_t s, uint32_t samples, bool *empty) {
    WaveStart start;
    cudaError_t e = started(pr, s, &start);
    if (e == cudaSuccess) *empty = start.kept == 0u && start.next >= samples;
    return e;
}

inline cudaError_t mark(StageMarks *m, int stage, cudaStream_t stream) {
    if (!m) return cudaSuccess;
    if (m->used == m->events.size()) {
        cudaEvent_t e;
        cudaError_t err = cudaEventCreate(&e);
        if (err != cudaSuccess) return err;
        m->events.push_back(e);
        m->stage.push_back(kStageGap);
    }
    m->stage[m->used] = stage;
    return cudaEventRecord(m->events[m->used++], stream);
}

}  // namespace

}  // namespace sg
