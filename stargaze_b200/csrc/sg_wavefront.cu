// sg_wavefront.cu — the integrator in wavefront form.
//
// The per-pixel megakernel (sg_kernels.cu) keeps a whole path in registers
// and walks it to the end, so a warp's lanes idle while the longest path of
// the 32 finishes and every lane drags the code of every vertex kind
// through the instruction cache. Here a dispatch's samples become paths in
// a pool whose state lives in HBM (seven float4 planes per path, read and
// written as 16-byte vectors, consecutive paths in consecutive slots), and
// each iteration runs three small kernels over it:
//
//   extend    tops the pool up with new camera paths (16x16 pixel tiles,
//             8x4 per warp, as the megakernel orders its lanes), then finds
//             the closest hit, point disc and ring crossing of every live
//             path; splits the paths into a ring queue and a surface queue
//             and finishes those that escaped;
//   ring      ring events (next-event estimation through the slab, null or
//             scatter), for the ring queue only;
//   surface   emitter hits and surface vertices (next-event estimation,
//             ringshine, cosine bounce), for the surface queue only.
//
// The shade stages append surviving paths, compacted, to the other state
// buffer. Queues are appended with one atomic per CTA and round (warp
// ballots, then a CTA prefix), so the order within a CTA is the order of
// its input. A new camera path is built in registers and stored only if it
// survives its first extend. Finished paths write their radiance to a
// per-(sample, pixel) slot; resolve sums each pixel's samples in sample
// order and folds them into the compensated accumulation exactly as the
// megakernel does. Both integrators run the same per-path functions
// (sg_integrator.cuh) on the same random sequences; they differ only where
// the compiler fuses a shading multiply-add in one kernel and not in the
// other, a few ulps.
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

// ---------------------------------------------------------------------------
// Stages
// ---------------------------------------------------------------------------
// A: the host air's code and the surface styles are compiled in (frames
// with air or styled bodies run these).
template <bool L, bool F, bool A>
__global__ void __launch_bounds__(kThreads, SG_WAVE_EXTEND_MIN_BLOCKS) wave_extend(const __grid_constant__ TraceParams P,
                                                                            const __grid_constant__ WaveParams W,
                                                                            uint32_t t) {
    extern __shared__ float4 smem[];
    // Celestial frames take several paths per append (their work per path
    // is even; SG_WAVE_EXTEND_ITEMS); landscape frames one, so that a CTA's
    // last round is small when traversal costs differ (measured with four:
    // rings 59.5 -> 56.5 ms per step, terrain 455 -> 531 ms). Landscape frames keep the append
    // barrier although their quadtree walks differ in length: writing a
    // per-path kind instead and building the queues in a kernel of their
    // own let the warps of a CTA drift apart, and the terrain step went
    // from 450 to 513 ms (the barrier keeps neighbouring pixels' walks
    // through the same quadtree nodes at the same time, in L1).
    constexpr uint32_t kItems = L ? 1u : SG_WAVE_EXTEND_ITEMS;
    __shared__ AppendK<2, kItems> sm[2];
    WaveCounters *c = counters(W, t);
    // Paths the previous iteration kept occupy [0, kept); new samples of the
    // chunk fill the pool up to n.
    const uint32_t kept = c->cont, next = c->next;
    const uint32_t per_sample = padded_pixels(W);
    const uint32_t take = min(W.pool - kept, per_sample * W.chunk_samples - next);
    const uint32_t n = kept + take;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counters(W, t + 1u)->next = next + take;
        *counters(W, t + 2u) = WaveCounters{};
        W.progress[t % kProgressSlots] = make_uint2(kept, next);
    }
    if (blockIdx.x * kThreads * kItems >= n) return;
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    Forward<A> nograd;
    float4 *st = W.state[t & 1u];
    float4 *H = W.hits;
    uint32_t round = 0;
    // Each round a thread extends kItems paths (i = base + k * kThreads +
    // threadIdx.x), then the CTA appends them to the queues at once.
    for (uint32_t base = blockIdx.x * kThreads * kItems; base < n; base += gridDim.x * kThreads * kItems, ++round) {
      uint32_t ring_bits = 0, surface_bits = 0;
#pragma unroll 1
      for (uint32_t item = 0; item < kItems; ++item) {
        const uint32_t i = base + item * kThreads + threadIdx.x;
        bool ring = false, surface = false;
        if (i < n) {
            Path p;
            uint32_t slot = 0;
            const bool fresh = i >= kept;
            bool valid = true;
            Cull cull = kTestAll;
            if (fresh) {
                // Sample k of the chunk, numbered sample-major over the
                // padded tile grid; padding pixels are skipped.
                const uint32_t k = next + (i - kept);
                const uint32_t smp = k / per_sample;
                const uint32_t q = k - smp * per_sample;
                const uint32_t tile = q >> 8, within = q & 255u;
                const uint32_t warp = within >> 5, lane = within & 31u;
                const uint32_t x = (tile % W.tiles_x) * kTile + (warp & 1u) * 8u + (lane & 7u);
                const uint32_t y = (tile / W.tiles_x) * kTile + (warp >> 1) * 4u + (lane >> 3);
                valid = x < P.width && y < P.height;
                if (valid) {
                    const uint32_t pixel = y * P.width + x;
                    start_path(p, &P.s, K, pixel, x, y, W.chunk_first + smp);
                    slot = smp * P.width * P.height + pixel;
                    cull = camera_cull<false>(P, tile);
                }
            } else {
                slot = load_ray_part(st, W.pool, i, p);
            }
            // A continuation leaving the host air may be attenuated in
            // extend: it needs its throughput.
            const bool was_in_air = A && !fresh && p.in_air;
            if (was_in_air) {
                const float4 c = st[2 * W.pool + i];
                p.throughput = xyz4(c);
                p.previous_pdf = c.w;
            }
            if (valid) {
                Extension e;
                const bool alive = extend(S, K, p, nograd, e, cull);
                ring = alive && e.ring.index != kMiss;
                surface = alive && !ring && e.hit.index != kMiss;
                if (ring || surface) {
                    if (fresh) {
                        store_path(st, W.pool, i, p, slot);
                    } else {
                        st[1 * W.pool + i] = pack3u(p.ray.d, p.rng);
                        st[6 * W.pool + i] = make_float4(iteration_word(p), depth_word(p), __uint_as_float(slot),
                                                         __uint_as_float(p.ckpt));
                        if (was_in_air) st[2 * W.pool + i] = pack3(p.throughput, p.previous_pdf);
                    }
                    if (ring) H[1 * W.pool + i] = pack3(e.ring.p, e.ring.t);
                    else H[0 * W.pool + i] = pack3(e.hit.n, e.hit.t);
                    H[2 * W.pool + i] = make_float4(__uint_as_float(e.hit.index), __uint_as_float(e.ring.index),
                                                    e.hit.delta, e.disc_scale);
                } else {
                    // Ended at the iteration bound, or escaped (then the sky
                    // backdrop of an unscattered camera path, as
                    // surface_vertex's miss). A new path's radiance is still
                    // zero.
                    if (!fresh) load_radiance_part(st, W.pool, i, p);
                    if (alive && (P.sky_on || (A && p.sky_on_escape))) {
                        if (!fresh && !was_in_air) p.throughput = xyz4(st[2 * W.pool + i]);
                        // A sky-lit local surface's continuation sees the
                        // surface sky cache (pathtrace.wgsl:1497-1499).
                        if (A && p.sky_on_escape)
                            p.radiance = p.radiance + p.throughput * surface_sky_lookup(S, p.ray.d);
                        sky_miss(S, p);
                    }
                    W.results[slot] = finish_path(p);
                    if (W.sky_results) W.sky_results[slot] = pack3(p.backdrop, 0.0f);
                    if (W.ck.totals) checkpoint_total(W.ck, W.chunk_first, P.width * P.height, slot, p);
                }
            }
        }
        ring_bits |= (ring ? 1u : 0u) << item;
        surface_bits |= (surface ? 1u : 0u) << item;
      }
      const uint32_t flags[2] = {ring_bits, surface_bits};
      uint32_t *const ctr[2] = {&c->ring, &c->surface};
      uint32_t q[2][kItems];
      block_append_k<2, kItems>(sm[round & 1u], flags, ctr, q);
#pragma unroll
      for (uint32_t item = 0; item < kItems; ++item) {
        const uint32_t i = base + item * kThreads + threadIdx.x;
        if ((ring_bits >> item) & 1u) W.ring_queue[q[0][item]] = i;
        if ((surface_bits >> item) & 1u) W.surface_queue[q[1][item]] = i;
      }
    }
}

// Ring (R == true) or surface stage over its queue. CK: the forward stores
// vertex checkpoints (W.ck). The ring stage runs at 3 CTAs per SM (85
// registers, fewer spills: 13.07 → 12.81 ms per 1080p ring step; 2 CTAs
// measured 13.57), the surface stage at 4 (3 measured slower).
template <bool L, bool F, bool R, bool A, bool CK = false>
__global__ void __launch_bounds__(kThreads, R ? 3 : SG_WAVE_SHADE_MIN_BLOCKS) wave_shade(const __grid_constant__ TraceParams P,
                                                                           const __grid_constant__ WaveParams W,
                                                                           uint32_t t) {
    extern __shared__ float4 smem[];
    constexpr int kQueues = CK ? 2 : 1;
    __shared__ Append<kQueues> sm[2];
    WaveCounters *c = counters(W, t);
    const uint32_t n = R ? c->ring : c->surface;
    if (blockIdx.x * kThreads >= n) return;
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    Stage<A> nograd;
    const float4 *st = W.state[t & 1u];
    float4 *out = W.state[(t + 1u) & 1u];
    const float4 *H = W.hits;
    const uint32_t *queue = R ? W.ring_queue : W.surface_queue;
    uint32_t round = 0;
    for (uint32_t base = blockIdx.x * kThreads; base < n; base += gridDim.x * kThreads, ++round) {
        const uint32_t j = base + threadIdx.x;
        bool keep = false, record = false;
        Path p;
        uint32_t slot = 0;
        if (j < n) {
            const uint32_t i = queue[j];
            slot = load_ray_part(st, W.pool, i, p);
            load_radiance_part(st, W.pool, i, p);
            load_shade_part(st, W.pool, i, p);
            const uint32_t depth_before = p.depth;
            const float4 h2 = H[2 * W.pool + i];
            bool ended;
            if constexpr (R) {
                const float4 h1 = H[1 * W.pool + i];
                const RingHit ring{h1.w, __float_as_uint(h2.y), xyz4(h1)};
                ended = ring_vertex(S, K, p, ring, nograd);
            } else {
                const float4 h0 = H[0 * W.pool + i];
                const Hit hit{h0.w, __float_as_uint(h2.x), h2.z, xyz4(h0)};
                ended = surface_vertex(S, K, p, hit, h2.w, nograd);
            }
            keep = !ended;
            if (ended) {
                W.results[slot] = finish_path(p);
                if (W.sky_results) W.sky_results[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (W.ck.totals) checkpoint_total(W.ck, W.chunk_first, P.width * P.height, slot, p);
            }
            if constexpr (CK) {
                // A scatter brought the depth to a checkpoint depth.
                record = keep && p.depth != depth_before && p.depth % W.ck.every == 0u && p.depth <= W.ck.max_depth &&
                         checkpoint_sample(W.ck, W.chunk_first, P.width * P.height, slot) < W.ck.samples;
            }
        }
        if constexpr (CK) {
            const bool flags[2] = {keep, record};
            uint32_t *const ctr[2] = {&counters(W, t + 1u)->cont, W.ck.count};
            uint32_t q[2];
            block_append<2>(sm[round & 1u], flags, ctr, q);
            if (record) {
                if (q[1] < W.ck.capacity) {
                    p.ckpt |= 1u;
                    const uint32_t pixels = P.width * P.height;
                    store_checkpoint(W.ck, q[1], p, slot % pixels, checkpoint_sample(W.ck, W.chunk_first, pixels, slot));
                } else {
                    p.ckpt |= 2u;
                }
            }
            if (keep) store_path(out, W.pool, q[0], p, slot);
        } else {
            const bool flags[1] = {keep};
            uint32_t *const ctr[1] = {&counters(W, t + 1u)->cont};
            uint32_t q[1];
            block_append<1>(sm[round & 1u], flags, ctr, q);
            if (keep) store_path(out, W.pool, q[0], p, slot);
        }
    }
}

// The tail of a chunk: once every sample is out and few paths are left,
// stage iterations cost their launches and load chains for a handful of
// paths each. Here every path live at the start of iteration t runs to its
// end in its own thread through the same per-path functions (step(), as
// the megakernel), and writes its result as the stages would.
template <bool L, bool F, bool A>
__global__ void __launch_bounds__(kThreads, SG_WAVE_SHADE_MIN_BLOCKS) wave_finish(const __grid_constant__ TraceParams P,
                                                                            const __grid_constant__ WaveParams W,
                                                                            uint32_t t) {
    extern __shared__ float4 smem[];
    const uint32_t n = counters(W, t)->cont;
    if (blockIdx.x * kThreads >= n) return;
    const Scene S = stage_scene(P, smem);
    const Counter<false, L, F> K{nullptr};
    Forward<A> nograd;
    const float4 *st = W.state[t & 1u];
#pragma unroll 1
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        Path p;
        const uint32_t slot = load_ray_part(st, W.pool, i, p);
        load_radiance_part(st, W.pool, i, p);
        load_shade_part(st, W.pool, i, p);
        p.backdrop = f3(0.0f, 0.0f, 0.0f);
        while (!step(S, K, p, nograd)) {
        }
        W.results[slot] = finish_path(p);
        if (W.sky_results) W.sky_results[slot] = pack3(p.backdrop, 0.0f);
        if (W.ck.totals) checkpoint_total(W.ck, W.chunk_first, P.width * P.height, slot, p);
    }
}

// Per pixel: the chunk's samples summed in sample order onto the running
// total, and on the last chunk the megakernel's compensated fold.
__global__ void __launch_bounds__(kThreads) wave_resolve(const __grid_constant__ TraceParams P,
                                                         const __grid_constant__ WaveParams W, int first, int last) {
    const uint32_t pixels = P.width * P.height;
    const uint32_t pixel = blockIdx.x * kThreads + threadIdx.x;
    if (pixel >= pixels) return;
    float4 total = first ? make_float4(0.0f, 0.0f, 0.0f, 0.0f) : W.totals[pixel];
    for (uint32_t smp = 0; smp < W.chunk_samples; ++smp) {
        const float4 r = W.results[(size_t)smp * pixels + pixel];
        total.x += r.x;
        total.y += r.y;
        total.z += r.z;
        total.w += r.w;
    }
    if (W.sky_results) {
        float3 sky = first ? f3(0.0f, 0.0f, 0.0f) : xyz4(W.sky_totals[pixel]);
        for (uint32_t smp = 0; smp < W.chunk_samples; ++smp) sky = sky + xyz4(W.sky_results[(size_t)smp * pixels + pixel]);
        if (last) fold_backdrop(P, pixel, sky);
        else W.sky_totals[pixel] = pack3(sky, 0.0f);
    }
    if (!last) {
        W.totals[pixel] = total;
        return;
    }
    const uint32_t old_count = P.s.counts[1];
    const float new_count = (float)(old_count + P.s.counts[2]);
    float4 sum, comp;
    if (old_count == 0u) {
        sum = total;
        comp = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    } else {
        sum = P.sum[pixel];
        comp = P.comp[pixel];
        float yv, tt;
        yv = __fsub_rn(total.x, comp.x); tt = __fadd_rn(sum.x, yv); comp.x = __fsub_rn(__fsub_rn(tt, sum.x), yv); sum.x = tt;
        yv = __fsub_rn(total.y, comp.y); tt = __fadd_rn(sum.y, yv); comp.y = __fsub_rn(__fsub_rn(tt, sum.y), yv); sum.y = tt;
        yv = __fsub_rn(total.z, comp.z); tt = __fadd_rn(sum.z, yv); comp.z = __fsub_rn(__fsub_rn(tt, sum.z), yv); sum.z = tt;
        yv = __fsub_rn(total.w, comp.w); tt = __fadd_rn(sum.w, yv); comp.w = __fsub_rn(__fsub_rn(tt, sum.w), yv); sum.w = tt;
    }
    P.sum[pixel] = sum;
    P.comp[pixel] = comp;
    P.mean[pixel] = make_float4(__fdiv_rn(__fsub_rn(sum.x, comp.x), new_count),
                                __fdiv_rn(__fsub_rn(sum.y, comp.y), new_count),
                                __fdiv_rn(__fsub_rn(sum.z, comp.z), new_count),
                                __fdiv_rn(__fsub_rn(sum.w, comp.w), new_count));
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct StageSet {
    const void *extend, *ring, *surface;
    const void *finish;  // null where vertex checkpoints are stored (their records need the stages' appends)
};

template <bool L, bool F, bool A, bool CK = false>
StageSet stage_set() {
    return StageSet{(const void *)wave_extend<L, F, A>, (const void *)wave_shade<L, F, true, A, CK>,
                    (const void *)wave_shade<L, F, false, A, CK>,
                    CK ? nullptr : (const void *)wave_finish<L, F, A>};
}

template <bool L, bool F, bool A>
cudaError_t run_finish(const TraceParams &p, const WaveParams &w, uint32_t t, uint32_t blocks, size_t smem,
                       cudaStream_t stream) {
    wave_finish<L, F, A><<<blocks, kThreads, smem, stream>>>(p, w, t);
    return cudaGetLastError();
}

// Live paths at or below which, once every sample of the chunk is out, the
// rest of the chunk runs in wave_finish (about one resident wave).
#ifndef SG_WAVE_FINISH_PATHS
#define SG_WAVE_FINISH_PATHS (1u << 18)
#endif
constexpr uint32_t kFinishPaths = SG_WAVE_FINISH_PATHS;

template <bool L, bool F, bool A, bool CK = false>
cudaError_t run_iteration(const TraceParams &p, const WaveParams &w, uint32_t t, const int (&grid)[4], size_t smem,
                          cudaStream_t stream, StageMarks *m) {
    cudaError_t e;
    if ((e = mark(m, kStageExtend, stream)) != cudaSuccess) return e;
    wave_extend<L, F, A><<<grid[0], kThreads, smem, stream>>>(p, w, t);
    if ((e = mark(m, kStageRing, stream)) != cudaSuccess) return e;
    wave_shade<L, F, true, A, CK><<<grid[1], kThreads, smem, stream>>>(p, w, t);
    if ((e = mark(m, kStageSurface, stream)) != cudaSuccess) return e;
    wave_shade<L, F, false, A, CK><<<grid[2], kThreads, smem, stream>>>(p, w, t);
    if ((e = mark(m, kStageGap, stream)) != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace

size_t wave_state_bytes(uint32_t pool) {
    return (size_t)pool * sizeof(float4) * (2 * kWavePlanes + kWaveHitPlanes) + (size_t)pool * 2 * sizeof(uint32_t) +
           kWaveCounterSets * sizeof(WaveCounters);
}

size_t wave_result_bytes(uint32_t pixels, uint32_t chunk_samples) {
    return (size_t)pixels * sizeof(float4) * ((size_t)chunk_samples + 1u);
}

cudaError_t launch_wavefront(const TraceParams &p, WaveParams w, WaveProgress &progress, cudaStream_t stream,
                             WaveRun *run, StageMarks *marks) {
    const uint32_t z = p.s.counts[2];
    const uint32_t pixels = p.width * p.height;
    *run = WaveRun{};
    if (marks) marks->used = 0;
    if (z == 0 || pixels == 0) return cudaSuccess;
    const bool land = p.s.g.ground_north[3] != 0.0f;
    // Checkpoints are stored for the frames the adjoint differentiates
    // (no air, no styles): variants 8-11.
    const bool ck = w.ck.records != nullptr;
    if (ck && (p.air_on || p.styled)) return cudaErrorInvalidValue;
    const int variant = (ck ? 8 : 0) | (p.air_on || p.styled ? 4 : 0) | (land ? 2 : 0) | (p.fp64_sites ? 1 : 0);
    StageSet set;
    switch (variant) {
        case 0: set = stage_set<false, false, false>(); break;
        case 1: set = stage_set<false, true, false>(); break;
        case 2: set = stage_set<true, false, false>(); break;
        case 3: set = stage_set<true, true, false>(); break;
        case 4: set = stage_set<false, false, true>(); break;
        case 5: set = stage_set<false, true, true>(); break;
        case 6: set = stage_set<true, false, true>(); break;
        case 7: set = stage_set<true, true, true>(); break;
        case 8: set = stage_set<false, false, false, true>(); break;
        case 9: set = stage_set<false, true, false, true>(); break;
        case 10: set = stage_set<true, false, false, true>(); break;
        default: set = stage_set<true, true, false, true>(); break;
    }
    const size_t smem = trace_smem_bytes(p);
    const void *fns[4] = {set.extend, set.ring, set.surface, set.finish};
    int grid[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) {
        if (!fns[k]) continue;
        const size_t bytes = smem;
        if (bytes > 48u * 1024u) {
            cudaError_t e = cudaFuncSetAttribute(fns[k], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
            if (e != cudaSuccess) return e;
        }
        cudaError_t e = persistent_grid(fns[k], bytes, &grid[k]);
        if (e != cudaSuccess) return e;
    }
    w.tiles_x = (p.width + kTile - 1) / kTile;
    w.tiles_y = (p.height + kTile - 1) / kTile;
    const uint32_t chunk = w.chunk_samples;
    const uint32_t per_sample = w.tiles_x * w.tiles_y * 256u;
    // A path ends within max_vertices * (bodies + 2) + 1 iterations, and an
    // iteration that takes no new sample has a full pool of paths that all
    // advance, so a chunk drains within (samples + 1) * (that + 1)
    // iterations: a host-side guard.
    const uint64_t cap = (uint64_t)p.s.counts[3] * (p.s.counts[0] + 2u) + 2u;
    for (uint32_t first = 0; first < z; first += chunk) {
        w.chunk_first = first;
        w.chunk_samples = std::min(chunk, z - first);
        const uint32_t samples = per_sample * w.chunk_samples;
        const uint64_t bound = ((uint64_t)samples + 1u) * cap;
        cudaError_t e = cudaMemsetAsync(w.counters, 0, kWaveCounterSets * sizeof(WaveCounters), stream);
        if (e != cudaSuccess) return e;
        // The host reads the start of iteration t - kLookahead while the
        // GPU runs the later ones; once one started empty the chunk has
        // drained (the iterations after it are empty launches).
        for (uint64_t t = 0;; ++t) {
            if (t >= bound) return cudaErrorLaunchTimeout;
            const uint32_t it = (uint32_t)t;
            switch (variant) {
                case 0: e = run_iteration<false, false, false>(p, w, it, grid, smem, stream, marks); break;
                case 1: e = run_iteration<false, true, false>(p, w, it, grid, smem, stream, marks); break;
                case 2: e = run_iteration<true, false, false>(p, w, it, grid, smem, stream, marks); break;
                case 3: e = run_iteration<true, true, false>(p, w, it, grid, smem, stream, marks); break;
                case 4: e = run_iteration<false, false, true>(p, w, it, grid, smem, stream, marks); break;
                case 5: e = run_iteration<false, true, true>(p, w, it, grid, smem, stream, marks); break;
                case 6: e = run_iteration<true, false, true>(p, w, it, grid, smem, stream, marks); break;
                case 7: e = run_iteration<true, true, true>(p, w, it, grid, smem, stream, marks); break;
                case 8: e = run_iteration<false, false, false, true>(p, w, it, grid, smem, stream, marks); break;
                case 9: e = run_iteration<false, true, false, true>(p, w, it, grid, smem, stream, marks); break;
                case 10: e = run_iteration<true, false, false, true>(p, w, it, grid, smem, stream, marks); break;
                default: e = run_iteration<true, true, false, true>(p, w, it, grid, smem, stream, marks); break;
            }
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
            if (set.finish && start.next >= samples && start.kept <= kFinishPaths) {
                const uint32_t blocks = std::min<uint32_t>(grid[3], (start.kept + kThreads - 1) / kThreads);
                if (blocks > 0u) {
                    if ((e = mark(marks, kStageFinish, stream)) != cudaSuccess) return e;
                    switch (variant) {
                        case 0: e = run_finish<false, false, false>(p, w, it + 1u, blocks, smem, stream); break;
                        case 1: e = run_finish<false, true, false>(p, w, it + 1u, blocks, smem, stream); break;
                        case 2: e = run_finish<true, false, false>(p, w, it + 1u, blocks, smem, stream); break;
                        case 3: e = run_finish<true, true, false>(p, w, it + 1u, blocks, smem, stream); break;
                        case 4: e = run_finish<false, false, true>(p, w, it + 1u, blocks, smem, stream); break;
                        case 5: e = run_finish<false, true, true>(p, w, it + 1u, blocks, smem, stream); break;
                        case 6: e = run_finish<true, false, true>(p, w, it + 1u, blocks, smem, stream); break;
                        default: e = run_finish<true, true, true>(p, w, it + 1u, blocks, smem, stream); break;
                    }
                    if (e != cudaSuccess) return e;
                    if ((e = mark(marks, kStageGap, stream)) != cudaSuccess) return e;
                    run->kernels += 1;
                }
                break;
            }
        }
        const bool first_chunk = first == 0, last_chunk = first + w.chunk_samples >= z;
        if ((e = mark(marks, kStageResolve, stream)) != cudaSuccess) return e;
        wave_resolve<<<(pixels + kThreads - 1) / kThreads, kThreads, 0, stream>>>(p, w, first_chunk, last_chunk);
        if ((e = mark(marks, kStageGap, stream)) != cudaSuccess) return e;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        run->kernels += 1;
    }
    return cudaSuccess;
}

}  // namespace sg
