// sg_wave_adjoint.cu — the path-replay adjoint in stages.
//
// The per-pixel adjoint (adjoint_kernel, sg_kernels.cu) replays each sample
// in one thread with every derivative hook inlined into the integrator, and
// is bound by instruction fetch as the forward megakernel was. Here the
// replay runs through the wavefront's stages (sg_wavefront.cu): extend over
// all live paths, ring_vertex over the ring queue, surface_vertex over the
// surface queue, the hooks of sg_adjoint.cuh running inside each.
//
// Each path holds an adjoint slot from its first surviving extend to its
// end: ten float4 of persistent state (running weighted sum, cap record,
// flags, and pass 2's weights) plus its PrbLists (Russian-roulette records
// after the cap vertex, deferred factors). Slots are taken from and given
// back to a ring of free slot ids. At the end of pass 1 a path either
// scatters its deferred factors and gives its slot back, or — when the
// ring-indirect cap binds or its deferral list overflowed — sets up pass 2
// in the same slot and restarts from its camera ray in the next iteration,
// exactly the two replays of the per-pixel adjoint. Gradients land in the
// same sinks: per-thread sums for the first bodies' colours, shared-memory
// windows over the ring tables and colours, global atomics for the rest,
// flushed at the end of every stage launch.
#include <algorithm>

// The stage kernels are small enough to inline the multi-site helpers and
// the derivative hooks that the per-pixel kernels keep out of line for
// their instruction footprint (measured on the ring workload: forward 6 %,
// adjoint 14 % faster inlined).
#define SG_HELPER __forceinline__
#define SG_ADJ_HOOK __forceinline__

#include "sg_wave_common.cuh"

namespace sg {

namespace {

// Resident CTAs per SM the stages are compiled for. The extend stage keeps
// the adjoint state out of its main loop (extend_end), so it fits the
// forward's register budget.
#ifndef SG_WAVE_ADJ_EXTEND_MIN_BLOCKS
#define SG_WAVE_ADJ_EXTEND_MIN_BLOCKS 4
#endif
#ifndef SG_WAVE_ADJ_SHADE_MIN_BLOCKS
#define SG_WAVE_ADJ_SHADE_MIN_BLOCKS 2
#endif
// CTA size of the shade stages. Smaller CTAs wait at each queue append for
// fewer slow warps but measured slower on the ring scene (64, 128, 256
// threads at 128 registers: 11.3, 10.3, 9.8 ms).
#ifndef SG_WAVE_ADJ_SHADE_THREADS
#define SG_WAVE_ADJ_SHADE_THREADS 256
#endif
constexpr int kShadeThreads = SG_WAVE_ADJ_SHADE_THREADS;
// Live paths at or below which, once every sample is out, the rest of the
// replay runs in adj_finish (about one resident wave of its threads).
#ifndef SG_ADJ_FINISH_PATHS
#define SG_ADJ_FINISH_PATHS (1u << 18)
#endif
constexpr uint32_t kFinishPaths = SG_ADJ_FINISH_PATHS;

// Slot state (float4 words):
//   0  a.xyz, cap                         5  w_pdf.xyz        (pass 2)
//   1  base.xyz, capture_iter             6  w_cap.xyz        (pass 2)
//   2  cap_light.xyz, flags               7  b.xyz            (pass 2)
//   3  prev_param, prev_dlog_pdf,         8  a_total.xyz      (pass 2)
//      score, sample index                9  b_total.xyz      (pass 2)
//   4  w_post.xyz (pass 2)
// flags: n_fac | n_rr << 8 | deferral_full, cap_direct, binding, pass 2.
constexpr uint32_t kFlagDeferralFull = 1u << 16;
constexpr uint32_t kFlagCapDirect = 1u << 17;
constexpr uint32_t kFlagBinding = 1u << 18;
constexpr uint32_t kFlagPass2 = 1u << 19;
// The forward stored the sample's radiance (sg_set_checkpoints): one
// replay scatters everything at once (segment_setup); with kFlagStops the
// replay ends where the first vertex checkpoint starts (the segment kernel
// replays the rest).
constexpr uint32_t kFlagKnownTotal = 1u << 20;
constexpr uint32_t kFlagStops = 1u << 21;

// Returns the slot's flags word.
__device__ __forceinline__ uint32_t load_prb(const AdjointWave &X, uint32_t slot, float3 w, Prb &G, uint32_t &smp) {
    const float4 *q = X.side + (size_t)slot * kAdjointSideVec4;
    const float4 s0 = q[0], s1 = q[1], s2 = q[2], s3 = q[3];
    const uint32_t flags = __float_as_uint(s2.w);
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    G.pass2 = (flags & kFlagPass2) != 0u;
    G.known_total = (flags & kFlagKnownTotal) != 0u;
    G.a = xyz4(s0);
    G.cap = s0.w;
    G.base = xyz4(s1);
    G.capture_iter = __float_as_uint(s1.w);
    G.cap_light = xyz4(s2);
    G.n_fac = flags & 0xffu;
    G.n_rr = (flags >> 8) & 0xffu;
    G.deferral_full = (flags & kFlagDeferralFull) != 0u;
    G.cap_direct = (flags & kFlagCapDirect) != 0u;
    G.binding = (flags & kFlagBinding) != 0u;
    G.prev_param = __float_as_uint(s3.x);
    G.prev_dlog_pdf = s3.y;
    G.score = s3.z;
    smp = __float_as_uint(s3.w);
    G.w_pre = w;
    if (G.pass2) {
        G.w_post = xyz4(q[4]);
        G.w_pdf = xyz4(q[5]);
        G.w_cap = xyz4(q[6]);
        G.b = xyz4(q[7]);
        G.a_total = xyz4(q[8]);
        G.b_total = xyz4(q[9]);
    } else {
        G.w_post = w;
        G.w_pdf = zero;
        G.w_cap = zero;
        G.b = zero;
        G.a_total = zero;
        G.b_total = zero;
    }
    G.lists = reinterpret_cast<PrbLists *>(X.lists) + slot;
    G.local = nullptr;  // the shade stages point it at their shared-memory lists
    G.local_stride = 0u;
    G.n_local = 0;
    G.dropped = 0;
    return flags;
}

__device__ __forceinline__ void store_prb(const AdjointWave &X, uint32_t slot, const Prb &G, uint32_t smp,
                                          uint32_t extra = 0u) {
    float4 *q = X.side + (size_t)slot * kAdjointSideVec4;
    const uint32_t flags = (G.n_fac & 0xffu) | ((G.n_rr & 0xffu) << 8) | (G.deferral_full ? kFlagDeferralFull : 0u) |
                           (G.cap_direct ? kFlagCapDirect : 0u) | (G.binding ? kFlagBinding : 0u) |
                           (G.pass2 ? kFlagPass2 : 0u) | (G.known_total ? kFlagKnownTotal : 0u) | extra;
    q[0] = pack3(G.a, G.cap);
    q[1] = pack3u(G.base, G.capture_iter);
    q[2] = pack3u(G.cap_light, flags);
    q[3] = make_float4(__uint_as_float(G.prev_param), G.prev_dlog_pdf, G.score, __uint_as_float(smp));
    if (G.pass2) {
        q[4] = pack3(G.w_post, 0.0f);
        q[5] = pack3(G.w_pdf, 0.0f);
        q[6] = pack3(G.w_cap, 0.0f);
        q[7] = pack3(G.b, 0.0f);
        q[8] = pack3(G.a_total, 0.0f);
        q[9] = pack3(G.b_total, 0.0f);
    }
}

// Pass 1's state of a new sample (pass1_setup) with the cap record cleared.
__device__ __forceinline__ void fresh_prb(Prb &G, float3 w) {
    pass1_setup(G, w);
    G.cap = 0.0f;
    G.base = f3(0.0f, 0.0f, 0.0f);
    G.cap_light = f3(0.0f, 0.0f, 0.0f);
    G.cap_direct = false;
    G.dropped = 0;
}

// The adjoint state of a sample that starts in this iteration, as its slot
// would hold it: pass 1 from the start, or — with the forward's radiance of
// the sample (sg_set_checkpoints) and no binding cap or overflowing record
// — one replay with every weight known (segment_setup), which ends at the
// first checkpoint when the sample has records (returns kFlagStops then).
__device__ __forceinline__ uint32_t fresh_sample(const TraceParams &P, const AdjointParams &A, const AdjointWave &X,
                                                 uint32_t slot, uint32_t pixel, uint32_t smp, float3 w, Prb &G) {
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    fresh_prb(G, w);
    G.a_total = zero;
    G.b_total = zero;
    G.lists = reinterpret_cast<PrbLists *>(X.lists) + slot;
    G.local = nullptr;
    G.local_stride = 0u;
    const uint32_t sample = A.ck.sample_base + smp;
    if (!A.ck.totals || sample >= A.ck.samples) return 0u;
    const float4 tot = A.ck.totals[(size_t)sample * P.width * P.height + pixel];
    const uint32_t bits = __float_as_uint(tot.w);
    if (bits & 2u) return 0u;
    segment_setup(G, w, f3(tot.x, tot.y, tot.z), zero);
    return (bits & 1u) ? kFlagStops : 0u;
}

// The pixel weight of the loss: d loss / d pixel over the samples behind it.
__device__ __forceinline__ float3 pixel_weight(const AdjointParams &A, uint32_t pixel) {
    const float4 d = A.dl_dimage[pixel];
    return f3(d.x, d.y, d.z) * A.inv_samples;
}

// Per-block gradient sinks: shared-memory windows over the ring tables and
// the body colours, and per-thread sums for the first bodies' colours in
// shared memory too (column threadIdx.x of a 6 kColorSlots x CTA-size
// block after the windows). In local memory those sums are read and
// written at every colour derivative, and at two 256-thread CTAs per SM
// the stages' local memory does not stay in L1.
struct BlockSink {
    float4 *inv;
    float *window;
    uint32_t window_n;
    float *own;     // this thread's column
    float4 *local;  // this thread's column of the pending-factor lists (shade stages)
};

__device__ __forceinline__ BlockSink open_sink(const TraceParams &P, const AdjointParams &A, float4 *smem) {
    const uint32_t n_bodies = P.s.counts[0];
    BlockSink b;
    b.inv = smem + trace_smem_floats(P) / 4u;
    b.window = reinterpret_cast<float *>(b.inv + 2u * n_bodies);
    b.window_n = A.tau_window + A.color_window;
    b.own = b.window + b.window_n + threadIdx.x;
    b.local = reinterpret_cast<float4 *>(b.window + ((b.window_n + 3u) & ~3u) + 6u * kColorSlots * blockDim.x) +
              threadIdx.x;
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) b.own[k * blockDim.x] = 0.0f;
    for (uint32_t k = threadIdx.x; k < b.window_n; k += blockDim.x) b.window[k] = 0.0f;
    for (uint32_t k = threadIdx.x; k < n_bodies; k += blockDim.x) {
        const float4 m = P.bodies[k * kBodyVec4 + kMaterial], r = P.bodies[k * kBodyVec4 + kRingColor];
        b.inv[2u * k] = make_float4(inv_or_zero(m.x), inv_or_zero(m.y), inv_or_zero(m.z), 0.0f);
        b.inv[2u * k + 1u] = make_float4(inv_or_zero(r.x), inv_or_zero(r.y), inv_or_zero(r.z), 0.0f);
    }
    return b;  // stage_scene's barrier publishes both
}

// Reduce the per-thread sums over the warp, then flush the windows.
__device__ __forceinline__ void close_sink(const AdjointParams &A, const BlockSink &b, unsigned long long dropped) {
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t k = 0; k < 6u * kColorSlots; ++k) {
        float v = b.own[k * blockDim.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0u && v != 0.0f) {
            if (k < A.color_window) atomicAdd(b.window + A.tau_window + k, v);
            else atomicAdd(A.grad + kGradColor + k, v);
        }
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < b.window_n; k += blockDim.x) {
        const float v = b.window[k];
        if (v != 0.0f) atomicAdd(A.grad + (k < A.tau_window ? k : kGradColor + (k - A.tau_window)), v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dropped += __shfl_down_sync(0xffffffffu, dropped, o);
    if (lane == 0u && dropped != 0ull && A.overflow) atomicAdd(A.overflow, dropped);
}

// End of a replay: pass 1 either scatters its deferred factors (the slot is
// then given back) or sets up pass 2 and restarts the sample from its camera
// ray; pass 2 just gives the slot back. Returns true on a restart.
template <bool L, bool F>
__device__ __forceinline__ bool end_replay(const TraceParams &P, Counter<false, L, F> K, Prb &G, Path &p,
                                           uint32_t pixel, uint32_t smp, float3 w) {
    if (G.pass2) return false;
    if (G.deferral_full || cap_binds(G, p.radiance)) {
        pass2_setup(G, p.radiance, w);
        start_path(p, &P.s, K, pixel, pixel % P.width, pixel / P.width, smp);
        return true;
    }
    flush_deferred(G);
    return false;
}

// A replay that ends at extend (escaped, or at the iteration bound) with
// path radiance `radiance`: loads its adjoint state and ends it. Returns
// the sample index in the low word when the sample restarts for pass 2 (the
// slot state is then stored), kMiss when the slot is given back; the high
// word counts dropped derivative entries. Everything is passed by value so
// that the caller's path stays in registers.
static __device__ __noinline__ unsigned long long extend_end(const AdjointParams &A, const AdjointWave &X,
                                                            GradSink sink, const float4 *inv, float3 radiance,
                                                            uint32_t iterations, uint32_t pixel, uint32_t slot) {
    const float3 w = pixel_weight(A, pixel);
    Prb G;
    uint32_t smp;
    load_prb(X, slot, w, G, smp);
    G.sink = sink;
    G.inv = inv;
    G.iteration = iterations;
    uint32_t code = kMiss;
    if (!G.pass2) {
        if (G.deferral_full || cap_binds(G, radiance)) {
            pass2_setup(G, radiance, w);
            store_prb(X, slot, G, smp);
            code = smp;
        } else {
            flush_deferred(G);
        }
    }
    return ((unsigned long long)G.dropped << 32) | code;
}

__device__ __forceinline__ float4 plane6(const Path &p, uint32_t pixel, uint32_t slot) {
    return make_float4(iteration_word(p), depth_word(p), __uint_as_float(pixel), __uint_as_float(slot));
}

// Stores every plane of a path whose plane 6 carries (pixel, slot).
__device__ __forceinline__ void store_adjoint_path(float4 *st, uint32_t pool, uint32_t i, const Path &p,
                                                   uint32_t pixel, uint32_t slot) {
    store_path(st, pool, i, p, 0u);
    st[6 * pool + i] = plane6(p, pixel, slot);
}

template <bool L, bool F>
__global__ void __launch_bounds__(kThreads, SG_WAVE_ADJ_EXTEND_MIN_BLOCKS)
    adj_extend(const __grid_constant__ TraceParams P, const __grid_constant__ AdjointParams A,
               const __grid_constant__ WaveParams W, const __grid_constant__ AdjointWave X, uint32_t t) {
    extern __shared__ float4 smem[];
    __shared__ Append<5> sm[2];
    WaveCounters *c = counters(W, t);
    const uint32_t kept = c->cont, next = c->next;
    const uint32_t per_sample = padded_pixels(W);
    const uint32_t take = min(W.pool - kept, per_sample * W.chunk_samples - next);
    const uint32_t n = kept + take;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters(W, t + 1u)->next = next + take;
        *counters(W, t + 2u) = WaveCounters{};
        W.progress[t % kProgressSlots] = make_uint2(kept, next);
    }
    if (blockIdx.x * kThreads >= n) return;
    const BlockSink bs = open_sink(P, A, smem);
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    const uint32_t n_bodies = P.s.counts[0];
    const uint32_t own_n = 6u * (n_bodies < kColorSlots ? n_bodies : kColorSlots);
    const GradSink sink{bs.own, own_n, bs.window, A.tau_window, bs.window + A.tau_window, A.color_window, A.grad,
                        blockDim.x};
    unsigned long long dropped = 0;
    float4 *st = W.state[t & 1u];
    float4 *out = W.state[(t + 1u) & 1u];
    float4 *H = W.hits;
    uint32_t round = 0;
    for (uint32_t base = blockIdx.x * kThreads; base < n; base += gridDim.x * kThreads, ++round) {
        const uint32_t i = base + threadIdx.x;
        bool ring = false, surface = false, restart = false, give = false, take_slot = false;
        Path p;
        Extension e;
        uint32_t pixel = 0, slot = 0, smp = 0;
        float3 w = f3(0.0f, 0.0f, 0.0f);
        const bool fresh = i >= kept;
        Cull cull = kTestAll;
        if (i < n) {
            bool valid = true;
            if (fresh) {
                const uint32_t k = next + (i - kept);
                smp = k / per_sample;
                const uint32_t q = k - smp * per_sample;
                const uint32_t tile = q >> 8, within = q & 255u;
                const uint32_t warp = within >> 5, lane = within & 31u;
                const uint32_t x = (tile % W.tiles_x) * kTile + (warp & 1u) * 8u + (lane & 7u);
                const uint32_t y = (tile / W.tiles_x) * kTile + (warp >> 1) * 4u + (lane >> 3);
                valid = x < P.width && y < P.height;
                if (valid) {
                    pixel = y * P.width + x;
                    w = pixel_weight(A, pixel);
                    // Pixels the loss does not weigh are not replayed.
                    valid = w.x != 0.0f || w.y != 0.0f || w.z != 0.0f;
                }
                if (valid) {
                    start_path(p, &P.s, K, pixel, x, y, smp);
                    cull = camera_cull<false>(P, tile);
                }
            } else {
                load_ray_part(st, W.pool, i, p);
                const float4 g = st[6 * W.pool + i];
                pixel = __float_as_uint(g.z);
                slot = __float_as_uint(g.w);
            }
            if (valid) {
                NoGrad nograd;  // extend's only hook sets the iteration
                const bool alive = extend(S, K, p, nograd, e, cull);
                ring = alive && e.ring.index != kMiss;
                surface = alive && !ring && e.hit.index != kMiss;
                take_slot = fresh && (ring || surface);
                if (!fresh && !ring && !surface) {
                    // Escaped or at the iteration bound: the replay ends.
                    const float3 radiance = xyz4(st[3 * W.pool + i]);
                    const unsigned long long end =
                        extend_end(A, X, sink, bs.inv, radiance, p.iterations, pixel, slot);
                    dropped += end >> 32;
                    const uint32_t code = (uint32_t)end;
                    restart = code != kMiss;
                    give = !restart;
                    if (restart) start_path(p, &P.s, K, pixel, pixel % P.width, pixel / P.width, code);
                }
            }
        }
        const bool flags[5] = {ring, surface, restart, give, take_slot};
        uint32_t *const ctr[5] = {&c->ring, &c->surface, &counters(W, t + 1u)->cont, X.free_ends + 1,
                                  X.free_ends + 0};
        uint32_t q[5];
        block_append<5>(sm[round & 1u], flags, ctr, q);
        if (take_slot) {
            // The slot's state is set up by the shade stage (fresh_sample).
            // Allocation j takes slot j while j < pool, then the slot that
            // give-back j - pool wrote (in an earlier launch: a launch's
            // fresh paths fit in the slots free at its start).
            slot = q[4] < W.pool ? q[4] : X.free_ring[q[4] % W.pool];
            store_adjoint_path(st, W.pool, i, p, pixel, slot);
        } else if (ring || surface) {
            st[1 * W.pool + i] = pack3u(p.ray.d, p.rng);
            st[6 * W.pool + i] = plane6(p, pixel, slot);
        }
        if (ring || surface) {
            if (ring) H[1 * W.pool + i] = pack3(e.ring.p, e.ring.t);
            else H[0 * W.pool + i] = pack3(e.hit.n, e.hit.t);
            H[2 * W.pool + i] = make_float4(__uint_as_float(e.hit.index), __uint_as_float(e.ring.index), e.hit.delta,
                                            e.disc_scale);
            const uint32_t at = ring ? q[0] : W.pool + q[1];
            if (ring) W.ring_queue[q[0]] = i;
            else W.surface_queue[q[1]] = i;
            X.queued[at] = make_uint4(slot, pixel, smp, take_slot ? 1u : 0u);
        }
        if (restart) store_adjoint_path(out, W.pool, q[2], p, pixel, slot);
        if (give) X.free_ring[q[3] % W.pool] = slot;
    }
    close_sink(A, bs, dropped);
}

// Ring (R == true) or surface stage of the replay over its queue.
template <bool L, bool F, bool R>
__global__ void __launch_bounds__(kShadeThreads, SG_WAVE_ADJ_SHADE_MIN_BLOCKS)
    adj_shade(const __grid_constant__ TraceParams P, const __grid_constant__ AdjointParams A,
              const __grid_constant__ WaveParams W, const __grid_constant__ AdjointWave X, uint32_t t) {
    extern __shared__ float4 smem[];
    __shared__ Append<2, kShadeThreads> sm[2];
    WaveCounters *c = counters(W, t);
    const uint32_t n = R ? c->ring : c->surface;
    if (blockIdx.x * kShadeThreads >= n) return;
    const BlockSink bs = open_sink(P, A, smem);
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    const uint32_t n_bodies = P.s.counts[0];
    const uint32_t own_n = 6u * (n_bodies < kColorSlots ? n_bodies : kColorSlots);
    const GradSink sink{bs.own, own_n, bs.window, A.tau_window, bs.window + A.tau_window, A.color_window, A.grad,
                        blockDim.x};
    unsigned long long dropped = 0;
    const float4 *st = W.state[t & 1u];
    float4 *out = W.state[(t + 1u) & 1u];
    const float4 *H = W.hits;
    const uint32_t *queue = R ? W.ring_queue : W.surface_queue;
    uint32_t round = 0;
    for (uint32_t base = blockIdx.x * kShadeThreads; base < n; base += gridDim.x * kShadeThreads, ++round) {
        const uint32_t j = base + threadIdx.x;
        bool keep = false, give = false;
        Path p;
        Prb G;
        uint32_t pixel = 0, slot = 0, smp = 0;
        uint32_t stops = 0u;
        if (j < n) {
            // The path and its slot, pixel and sample come from the queue
            // entry, so that the slot state, the pixel weight and the path
            // state are read at once.
            const uint32_t i = queue[j];
            const uint4 entry = X.queued[(R ? 0u : W.pool) + j];
            slot = entry.x;
            pixel = entry.y;
            load_ray_part(st, W.pool, i, p);
            load_radiance_part(st, W.pool, i, p);
            load_shade_part(st, W.pool, i, p);
            const float3 w = pixel_weight(A, pixel);
            if (entry.w) {
                smp = entry.z;
                stops = fresh_sample(P, A, X, slot, pixel, smp, w, G);
            } else {
                stops = load_prb(X, slot, w, G, smp) & kFlagStops;
            }
            G.sink = sink;
            G.inv = bs.inv;
            G.local = bs.local;
            G.local_stride = blockDim.x;
            G.iteration = p.iterations;
            const float4 h2 = H[2 * W.pool + i];
            bool ended;
            if constexpr (R) {
                const float4 h1 = H[1 * W.pool + i];
                const RingHit ring{h1.w, __float_as_uint(h2.y), xyz4(h1)};
                ended = ring_vertex(S, K, p, ring, G);
            } else {
                const float4 h0 = H[0 * W.pool + i];
                const Hit hit{h0.w, __float_as_uint(h2.x), h2.z, xyz4(h0)};
                ended = surface_vertex(S, K, p, hit, h2.w, G);
            }
            keep = !ended || end_replay(P, K, G, p, pixel, smp, w);
            // A checkpointed sample's replay ends where its first record
            // starts (the same scatter that stored it in the forward).
            if (keep && !ended && G.known_total && p.depth >= A.ck.every && stops) keep = false;
            give = !keep;
            dropped += G.dropped;
        }
        const bool flags[2] = {keep, give};
        uint32_t *const ctr[2] = {&counters(W, t + 1u)->cont, X.free_ends + 1};
        uint32_t q[2];
        block_append<2, kShadeThreads>(sm[round & 1u], flags, ctr, q);
        if (keep) {
            store_prb(X, slot, G, smp, G.known_total ? stops : 0u);
            store_adjoint_path(out, W.pool, q[0], p, pixel, slot);
        }
        if (give) X.free_ring[q[1] % W.pool] = slot;
    }
    close_sink(A, bs, dropped);
}

// The tail of the replay: once every sample is out and few paths are left
// (mostly second replays of samples whose cap binds, a fraction of a
// percent), stage iterations cost their launches and load chains for a
// handful of paths each. Here every path live at the start of iteration t
// runs to its end in its own thread — the remaining vertices, and the
// second replay if its first ends on a binding cap — through the same
// per-path functions and hooks; no queues, no barriers.
template <bool L, bool F>
__global__ void __launch_bounds__(kShadeThreads, SG_WAVE_ADJ_SHADE_MIN_BLOCKS)
    adj_finish(const __grid_constant__ TraceParams P, const __grid_constant__ AdjointParams A,
               const __grid_constant__ WaveParams W, const __grid_constant__ AdjointWave X, uint32_t t) {
    extern __shared__ float4 smem[];
    const uint32_t n = counters(W, t)->cont;
    if (blockIdx.x * kShadeThreads >= n) return;
    const BlockSink bs = open_sink(P, A, smem);
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    const uint32_t n_bodies = P.s.counts[0];
    const uint32_t own_n = 6u * (n_bodies < kColorSlots ? n_bodies : kColorSlots);
    const GradSink sink{bs.own, own_n, bs.window, A.tau_window, bs.window + A.tau_window, A.color_window, A.grad,
                        blockDim.x};
    unsigned long long dropped = 0;
    const float4 *st = W.state[t & 1u];
#pragma unroll 1
    for (uint32_t i = blockIdx.x * kShadeThreads + threadIdx.x; i < n; i += gridDim.x * kShadeThreads) {
        Path p;
        load_ray_part(st, W.pool, i, p);
        load_radiance_part(st, W.pool, i, p);
        load_shade_part(st, W.pool, i, p);
        const float4 g = st[6 * W.pool + i];
        const uint32_t pixel = __float_as_uint(g.z), slot = __float_as_uint(g.w);
        const float3 w = pixel_weight(A, pixel);
        Prb G;
        uint32_t smp;
        const uint32_t stops = load_prb(X, slot, w, G, smp) & kFlagStops;
        G.sink = sink;
        G.inv = bs.inv;
        G.local = bs.local;
        G.local_stride = blockDim.x;
#pragma unroll 1
        for (;;) {
            const bool ended = step(S, K, p, G);
            if (!ended) {
                // A checkpointed sample's replay ends where its first record
                // starts (the segment kernel replays the rest).
                if (G.known_total && stops && p.depth >= A.ck.every) break;
                continue;
            }
            if (!end_replay(P, K, G, p, pixel, smp, w)) break;
        }
        dropped += G.dropped;
    }
    close_sink(A, bs, dropped);
}

template <bool L, bool F>
cudaError_t run_adjoint_iteration(const TraceParams &p, const AdjointParams &a, const WaveParams &w,
                                  const AdjointWave &x, uint32_t t, const int (&grid)[3], const size_t (&smem)[2],
                                  cudaStream_t stream) {
    adj_extend<L, F><<<grid[0], kThreads, smem[0], stream>>>(p, a, w, x, t);
    adj_shade<L, F, true><<<grid[1], kShadeThreads, smem[1], stream>>>(p, a, w, x, t);
    adj_shade<L, F, false><<<grid[2], kShadeThreads, smem[1], stream>>>(p, a, w, x, t);
    return cudaGetLastError();
}

}  // namespace

size_t adjoint_slot_bytes(uint32_t pool) {
    return (size_t)pool * (kAdjointSideVec4 * sizeof(float4) + 2u * sizeof(uint4) + sizeof(PrbLists)) +
           (size_t)pool * sizeof(uint32_t) + 4 * sizeof(uint32_t);
}

cudaError_t reset_adjoint_slots(const AdjointWave &x, uint32_t, cudaStream_t stream) {
    return cudaMemsetAsync(x.free_ends, 0, 2 * sizeof(uint32_t), stream);
}

cudaError_t launch_adjoint_wavefront(const TraceParams &p, const AdjointParams &a, WaveParams w,
                                     const AdjointWave &x, WaveProgress &progress, cudaStream_t stream, WaveRun *run) {
    *run = WaveRun{};
    const uint32_t z = p.s.counts[2];
    if (z == 0 || p.width == 0 || p.height == 0) return cudaSuccess;
    const bool land = p.s.g.ground_north[3] != 0.0f;
    const void *fns[3];
    if (land) {
        fns[0] = p.fp64_sites ? (const void *)adj_extend<true, true> : (const void *)adj_extend<true, false>;
        fns[1] = p.fp64_sites ? (const void *)adj_shade<true, true, true> : (const void *)adj_shade<true, false, true>;
        fns[2] = p.fp64_sites ? (const void *)adj_shade<true, true, false> : (const void *)adj_shade<true, false, false>;
    } else {
        fns[0] = p.fp64_sites ? (const void *)adj_extend<false, true> : (const void *)adj_extend<false, false>;
        fns[1] = p.fp64_sites ? (const void *)adj_shade<false, true, true> : (const void *)adj_shade<false, false, true>;
        fns[2] = p.fp64_sites ? (const void *)adj_shade<false, true, false> : (const void *)adj_shade<false, false, false>;
    }
    // After the adjoint's shared memory: the per-thread colour sums, and in
    // the shade stages the pending-factor lists (16-byte aligned).
    const size_t smem[2] = {
        adjoint_smem_bytes(p, a) + (size_t)6u * kColorSlots * kThreads * sizeof(float),
        adjoint_smem_bytes(p, a) + 16u + (size_t)6u * kColorSlots * kShadeThreads * sizeof(float) +
            (size_t)kMaxLocal * kShadeThreads * sizeof(float4)};
    int grid[3];
    for (int k = 0; k < 3; ++k) {
        const size_t bytes = smem[k == 0 ? 0 : 1];
        if (bytes > 48u * 1024u) {
            cudaError_t e = cudaFuncSetAttribute(fns[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = persistent_grid(fns[k], bytes, &grid[k], k == 0 ? kThreads : kShadeThreads);
        if (e != cudaSuccess) return e;
    }
    w.tiles_x = (p.width + kTile - 1) / kTile;
    w.tiles_y = (p.height + kTile - 1) / kTile;
    w.chunk_first = 0;
    w.chunk_samples = z;
    const uint32_t samples = w.tiles_x * w.tiles_y * 256u * z;
    // A sample replays at most twice, each replay ending within the
    // iteration bound; see launch_wavefront for the host-side guard.
    const uint64_t cap = 2ull * ((uint64_t)p.s.counts[3] * (p.s.counts[0] + 2u) + 2u);
    const uint64_t bound = ((uint64_t)samples + 1u) * cap;
    const void *finish = land ? (p.fp64_sites ? (const void *)adj_finish<true, true> : (const void *)adj_finish<true, false>)
                              : (p.fp64_sites ? (const void *)adj_finish<false, true>
                                              : (const void *)adj_finish<false, false>);
    int finish_grid = 0;
    if (smem[1] > 48u * 1024u) {
        cudaError_t e = cudaFuncSetAttribute(finish, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem[1]);
        if (e != cudaSuccess) return e;
    }
    if (cudaError_t e = persistent_grid(finish, smem[1], &finish_grid, kShadeThreads); e != cudaSuccess) return e;
    cudaError_t e = cudaMemsetAsync(w.counters, 0, kWaveCounterSets * sizeof(WaveCounters), stream);
    if (e != cudaSuccess) return e;
    for (uint64_t t = 0;; ++t) {
        if (t >= bound) return cudaErrorLaunchTimeout;
        const uint32_t it = (uint32_t)t;
        e = land ? (p.fp64_sites ? run_adjoint_iteration<true, true>(p, a, w, x, it, grid, smem, stream)
                                 : run_adjoint_iteration<true, false>(p, a, w, x, it, grid, smem, stream))
                 : (p.fp64_sites ? run_adjoint_iteration<false, true>(p, a, w, x, it, grid, smem, stream)
                                 : run_adjoint_iteration<false, false>(p, a, w, x, it, grid, smem, stream));
        if (e != cudaSuccess) return e;
        if ((e = iteration_done(progress, t, stream)) != cudaSuccess) return e;
        run->iterations += 1;
        run->kernels += 3;
        if (t < kLookahead) continue;
        WaveStart start;
        if ((e = started(progress, t - kLookahead, &start)) != cudaSuccess) return e;
        if (start.kept == 0u && start.next >= samples) break;
        // Every sample is out and few paths are left: no later iteration
        // holds more than iteration t - kLookahead did; finish them at once.
        if (start.next >= samples && start.kept <= kFinishPaths) {
            const uint32_t blocks = std::min<uint32_t>(finish_grid, (start.kept + kShadeThreads - 1) / kShadeThreads);
            const uint32_t next_t = it + 1u;
            if (blocks > 0u) {
                if (land) {
                    if (p.fp64_sites) adj_finish<true, true><<<blocks, kShadeThreads, smem[1], stream>>>(p, a, w, x, next_t);
                    else adj_finish<true, false><<<blocks, kShadeThreads, smem[1], stream>>>(p, a, w, x, next_t);
                } else {
                    if (p.fp64_sites) adj_finish<false, true><<<blocks, kShadeThreads, smem[1], stream>>>(p, a, w, x, next_t);
                    else adj_finish<false, false><<<blocks, kShadeThreads, smem[1], stream>>>(p, a, w, x, next_t);
                }
                if ((e = cudaGetLastError()) != cudaSuccess) return e;
                run->kernels += 1;
            }
            break;
        }
    }
    return cudaSuccess;
}

}  // namespace sg
