// sg_adjoint.cuh — derivative bookkeeping of the path-replay adjoint (an
// extension: stargaze renders forward only).
//
// The backward pass replays every sample of the accumulated image from its
// noise key, so each path takes exactly the forward's decisions. Sampling is
// detached: Russian roulette, the ring null-versus-scatter choice, point-disc
// picks, MIS weights and the pdfs that divide the estimator are held at
// their forward values, and only the integrand is differentiated. That
// keeps the estimator unbiased wherever the sampling pdf is positive:
// E[(df/dtheta) / p] is the derivative of the integral of f. (A ring bin at
// tau = 0 is never scattered in, so its gradient carries the transmission
// term only.)
//
// Path-replay backpropagation: a factor multiplied into the path throughput
// (surface albedo at a bounce, the slab BSDF at a ring scatter, the
// transmission of a null crossing) scales every radiance contribution after
// it, so its gradient is d log(factor) times the weighted radiance the path
// gathers from there on: A_total - A, where A is the running sum of
// w_c * c over the contributions c so far. A first replay of the sample
// (pass 1, no derivatives) finds A_total; the second (pass 2) scatters each
// factor once when it is created and each contribution's own factors
// (albedo of the shading point, emitted radiance of the light, slab BSDF at
// the ring point, ring transmissions along the shadow ray) when it is made.
// Most paths need only pass 1: it weighs every contribution by the pixel
// weight w — right unless the ring-indirect cap binds — scatters each
// contribution's own factors at once, and defers each throughput factor
// with the running sum A at its creation, scattering d log(factor) *
// (A_final - A) when the path ends. Only a path whose cap binds (or that
// overflows the deferral list) runs pass 2, which adds to the contributions
// after the cap vertex the difference between their weight and the w
// pass 1 gave them.
//
// The ring-indirect cap (pathtrace.wgsl:1609-1615) clamps the radiance I
// gathered after a path's first ring scatter to luminance `cap`:
// R = base + I * min(1, cap / lum(I)). The clamp makes R nonlinear in I, so
// on paths where it binds the detached form is biased. There the result is
// split into base + I (linear, detached) and C = I * (cap / lum(I) - 1),
// differentiated by the likelihood-ratio rule: the attached derivative of C
// (pdfs, Russian-roulette survivals and MIS weights varying with the
// parameters) plus C times the score — d log probability — of every
// decision from the cap vertex's scatter on. With s = cap / lum(I),
// w_c = (w . I) / lum(I) for the pixel weight w, the contribution weights
// are w before the cap vertex's scatter, s * (w - lum * w_c) after it
// (detached), that minus w for attached-only terms, lum * w_c for the cap's
// own luminance sum, and w . C for the scores. Pass 1 records the cap
// vertex, base, I, the cap sum and the Russian-roulette events after it.
//
// Parameters are indexed in the flat space of sg_internal.h (kGradColor,
// kGradMap). A parameter whose value is zero gets no gradient through its
// own log derivative.
#pragma once

#include "sg_device.cuh"
#include "sg_landscape.cuh"

// Call attribute of the derivative hooks: out of line by default, which
// keeps the per-pixel adjoint's instruction footprint to one replay.
#ifndef SG_ADJ_HOOK
#define SG_ADJ_HOOK __noinline__
#endif

namespace sg {

constexpr uint32_t kNoParam = 0xffffffffu;
constexpr uint32_t kVectorBit = 0x80000000u;  // entry spans an rgb triple
constexpr uint32_t kPdfBit = 0x40000000u;     // attached-only (scalar) entry
constexpr uint32_t kParamMask = 0x3fffffffu;
constexpr int kMaxRoulette = 6;               // recorded events after a cap vertex
constexpr int kMaxLocal = 8;                  // factors of one contribution
constexpr int kMaxCrossings = kMaxRecordedCrossings;  // of one shadow ray
constexpr uint32_t kColorSlots = 4;           // bodies with per-thread colour sums
constexpr int kMaxDeferred = 16;              // throughput factors pass 1 can defer

struct GradEntry {
    uint32_t param;  // kNoParam: none
    float3 dlog;     // scalar parameters use dlog.x for all channels
};

__device__ __forceinline__ GradEntry no_entry() { return GradEntry{kNoParam, make_float3(0.0f, 0.0f, 0.0f)}; }
__device__ __forceinline__ float4 pack_entry(const GradEntry &e) {
    return make_float4(__uint_as_float(e.param), e.dlog.x, e.dlog.y, e.dlog.z);
}
__device__ __forceinline__ GradEntry unpack_entry(float4 v) {
    return GradEntry{__float_as_uint(v.x), make_float3(v.y, v.z, v.w)};
}

// Where gradients land: the colours of the first kColorSlots bodies in
// per-thread sums (every lane of a warp hits the same few of them; the
// kernel reduces them once at its end), shared-memory windows over the
// ring tables in use and the other body colours, global memory for the
// rest. Sum k of a thread is own[k * own_stride]: a local array (stride 1)
// or the thread's column of a shared-memory block (stride: CTA size).
struct GradSink {
    float *own;         // per-thread sums over [kGradColor, kGradColor + own_n)
    uint32_t own_n;
    float *tau;
    uint32_t tau_n;
    float *color;
    uint32_t color_n;
    float *global;
    uint32_t own_stride;
    __device__ __forceinline__ void add(uint32_t param, float value) const {
        if (value == 0.0f) return;
        const uint32_t c = param - kGradColor;
        if (c < own_n) own[c * own_stride] += value;
        else if (param < tau_n) atomicAdd(tau + param, value);
        else if (c < color_n) atomicAdd(color + c, value);
        else atomicAdd(global + param, value);
    }
};

// The forward integrator: no hooks. A: the host air's code and the
// procedural surface styles are compiled in. Frames with air
// (atmo_params.w >= 0.5) or a styled body (axis_x.w >= 0.5) run the A
// instantiations; the others run kernels that carry none of that code or
// its register pressure.
template <bool A>
struct Forward {
    static constexpr bool adjoint = false;
    static constexpr bool sky = true;  // surface_vertex shades an escaped path's sky
    static constexpr bool air = A;
};
using NoGrad = Forward<false>;

// The wavefront's shade stages: no hooks, and no escaped paths (extend ends
// those), so surface_vertex's miss branch never runs there.
template <bool A>
struct Stage {
    static constexpr bool adjoint = false;
    static constexpr bool sky = false;
    static constexpr bool air = A;
};

// A Russian-roulette decision after the cap vertex (pathtrace.wgsl:
// 1484-1490, :1600-1604); its record (PrbLists::rr) also holds the radiance
// gathered since the cap vertex, before it.
struct Roulette {
    uint32_t iteration;
    uint32_t bits;  // max channel (0-2) | 4 survived | 8 survival clamped
    float s;        // survival probability
};

// The lists a path's adjoint appends to: Russian-roulette events after the
// cap vertex (with pass 2's coefficient of each) and pass 1's deferred
// throughput factors with the running sum at each. The per-pixel adjoint
// keeps them in the thread's local memory, the staged adjoint in a device
// slot that stays with the path across stages. Each entry is one 32-byte
// record (one DRAM sector in device memory, written whole):
//   fac[k]: (param, dlog.xyz), (running sum at the factor, 0)
//   rr[r]:  (iteration, bits, s, pass 2's coefficient), (before.xyz, 0)
struct PrbLists {
    float4 fac[kMaxDeferred][2];
    float4 rr[kMaxRoulette][2];
};

__device__ __forceinline__ Roulette roulette_at(const PrbLists *l, uint32_t r, float &coef) {
    const float4 a = l->rr[r][0];
    coef = a.w;
    return Roulette{__float_as_uint(a.x), __float_as_uint(a.y), a.z};
}

// The adjoint's state. Both passes run the same integrator code (one
// instantiation, so a warp's instruction footprint is that of one replay);
// pass 1 also records the summary pass 2 needs (`pass2` false).
struct Prb {
    static constexpr bool adjoint = true;
    static constexpr bool sky = false;  // sg_backward rejects frames with a sky
    static constexpr bool air = false;  // ... and frames with host air
    bool pass2;
    // A segment of a checkpointed path (sg_set_checkpoints): the path's total
    // is known from the forward, so one replay scatters everything at once
    // (contributions at full weight, factors with the radiance after them).
    bool known_total;
    // Pass 1's summary.
    float cap;
    float3 base;            // radiance at the cap vertex's scatter
    float3 cap_light;       // the rgb sum whose luminance is the cap
    float3 lit_sum, lit_vis_sum;  // at the current ring vertex
    // Pass 2.
    GradSink sink;
    const float4 *inv;        // per body: 1 / colour, 1 / ring colour
    float3 w_pre, w_post, w_pdf, w_cap;  // contribution weights (see above)
    float score;
    float3 a_total, b_total;  // weighted radiance of the whole path
    float3 a, b;              // ... gathered so far (detached, attached-only)
    uint32_t capture_iter;
    bool binding, cap_direct;
    uint32_t iteration;       // the current step's
    uint32_t prev_param;      // tau parameter of the last ring scatter
    float prev_dlog_pdf;      // ... and d log of its scatter pdf
    uint32_t n_rr;
    // The factors of the pending contribution: entry k at
    // local[k * local_stride] (a local array, stride 1, or the thread's
    // column of a shared-memory block), packed as float4.
    float4 *local;
    uint32_t local_stride;
    uint32_t n_local, dropped;
    // Pass 1's deferred throughput factors (count), and where the lists live.
    uint32_t n_fac;
    bool deferral_full;
    PrbLists *lists;

    __device__ __forceinline__ bool post() const { return capture_iter != 0u && iteration > capture_iter; }
    __device__ __forceinline__ bool after_capture() const { return capture_iter != 0u && iteration >= capture_iter; }
    __device__ __forceinline__ void local_factor(GradEntry e) {
        if (e.param == kNoParam) return;
        if (n_local < (uint32_t)kMaxLocal) local[(n_local++) * local_stride] = pack_entry(e);
        else dropped += 1u;
    }
};

__device__ __forceinline__ float inv_or_zero(float v) { return v != 0.0f ? 1.0f / v : 0.0f; }
__device__ __forceinline__ float3 inv3(float3 v) { return f3(inv_or_zero(v.x), inv_or_zero(v.y), inv_or_zero(v.z)); }
__device__ __forceinline__ float3 mul3(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float sum3(float3 a) { return a.x + a.y + a.z; }
__device__ __forceinline__ float channel(float3 v, uint32_t m) { return m == 0u ? v.x : (m == 1u ? v.y : v.z); }

__device__ __forceinline__ GradEntry vector_entry(uint32_t base, float3 dlog) {
    return GradEntry{base | kVectorBit, dlog};
}
__device__ __forceinline__ GradEntry scalar_entry(uint32_t param, float dlog) {
    return GradEntry{param, f3(dlog, dlog, dlog)};
}
__device__ __forceinline__ uint32_t ring_albedo_param(uint32_t body) { return kGradColor + 6u * body; }
__device__ __forceinline__ uint32_t body_color_param(uint32_t body) { return kGradColor + 6u * body + 3u; }

// Emitted radiance of a light (or an emitter hit): d log / d colour.
__device__ __forceinline__ GradEntry emitter_entry(const Prb &G, uint32_t body) {
    return vector_entry(body_color_param(body), xyz(G.inv[2u * body]));
}
__device__ __forceinline__ GradEntry ring_albedo_entry(const Prb &G, uint32_t body) {
    return vector_entry(ring_albedo_param(body), xyz(G.inv[2u * body + 1u]));
}

// Scatter `w . dlog` of one entry: per channel for a vector entry, the
// channel sum for a scalar one.
__device__ __forceinline__ void scatter_entry(const GradSink &sink, const GradEntry &e, float3 w, float3 w_pdf) {
    if (e.param & kPdfBit) {
        sink.add(e.param & kParamMask, sum3(w_pdf) * e.dlog.x);
    } else if (e.param & kVectorBit) {
        const uint32_t base = e.param & ~kVectorBit;
        sink.add(base + 0u, w.x * e.dlog.x);
        sink.add(base + 1u, w.y * e.dlog.y);
        sink.add(base + 2u, w.z * e.dlog.z);
    } else {
        sink.add(e.param, sum3(w) * e.dlog.x);
    }
}

// A radiance contribution `value` and its pending local factors (consumed).
// `cap_term`: the cap vertex's light sample as a term of the cap.
// Pass 1 scattered every contribution's local factors with weight w, so
// pass 2 scatters only what differs: nothing before the cap vertex's
// scatter, w_post - w after it, and the cap terms and attached entries in
// full. The running sums take each contribution's full weight.
static __device__ SG_ADJ_HOOK void contribute(Prb &G, float3 value, bool cap_term) {
    const bool post = G.post();
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    const float3 full = cap_term ? G.w_cap : (post ? G.w_post : G.w_pre);
    const float3 local =
        (!G.pass2 || G.known_total) ? full : (cap_term ? G.w_cap : (post ? G.w_post - G.w_pre : zero));
    const float3 w = mul3(local, value);
    const float3 wp = (!cap_term && post) ? mul3(G.w_pdf, value) : zero;
    if (w.x != 0.0f || w.y != 0.0f || w.z != 0.0f || wp.x != 0.0f || wp.y != 0.0f || wp.z != 0.0f) {
#pragma unroll 1
        for (uint32_t k = 0; k < G.n_local; ++k) scatter_entry(G.sink, unpack_entry(G.local[k * G.local_stride]), w, wp);
    }
    G.n_local = 0;
    G.a = G.a + mul3(full, value);
    G.b = G.b + wp;
}

// A factor multiplied into the throughput now: its share of everything the
// path gathers from here on, plus — past a binding cap vertex — its part in
// the later Russian-roulette survivals (score and attached 1 / s).
static __device__ SG_ADJ_HOOK void factor(Prb &G, GradEntry e) {
    if (e.param == kNoParam) return;
    if (!G.pass2) {
        // Pass 1: defer until the path's end.
        if (G.n_fac < (uint32_t)kMaxDeferred) {
            G.lists->fac[G.n_fac][0] = pack_entry(e);
            G.lists->fac[G.n_fac][1] = make_float4(G.a.x, G.a.y, G.a.z, 0.0f);
            G.n_fac += 1u;
        } else {
            G.deferral_full = true;
        }
        return;
    }
    const bool pdf = (e.param & kPdfBit) != 0u, vec = (e.param & kVectorBit) != 0u;
    float3 add;
    if (pdf) add = f3(sum3(G.b_total - G.b) * e.dlog.x, 0.0f, 0.0f);
    else if (vec) add = mul3(G.a_total - G.a, e.dlog);
    else add = f3(sum3(G.a_total - G.a) * e.dlog.x, 0.0f, 0.0f);
    if (G.binding) {
        // d log s of a survival s = clamp(t_m) is d log t_m: channel m of a
        // vector entry, the whole scalar entry for the first unclamped
        // survival (later ones see t / s, which no scalar factor moves).
        int prev = -1;
#pragma unroll 1
        for (uint32_t r = 0; r < G.n_rr; ++r) {
            float c;
            const Roulette ev = roulette_at(G.lists, r, c);
            if (ev.iteration < G.iteration || (ev.bits & 8u)) continue;
            const uint32_t m = ev.bits & 3u;
            if (vec) {
                const float dm = c * channel(e.dlog, m);
                add = f3(add.x + (m == 0u ? dm : 0.0f), add.y + (m == 1u ? dm : 0.0f), add.z + (m == 2u ? dm : 0.0f));
                if (prev >= 0) {
                    const float dp = c * channel(e.dlog, (uint32_t)prev);
                    add = f3(add.x - (prev == 0 ? dp : 0.0f), add.y - (prev == 1 ? dp : 0.0f),
                             add.z - (prev == 2 ? dp : 0.0f));
                }
            } else if (prev < 0) {
                add.x += c * e.dlog.x;
            }
            if (!(ev.bits & 4u)) break;
            prev = (int)m;
        }
    }
    if (vec) {
        const uint32_t base = e.param & ~kVectorBit;
        G.sink.add(base + 0u, add.x);
        G.sink.add(base + 1u, add.y);
        G.sink.add(base + 2u, add.z);
    } else {
        G.sink.add(e.param & kParamMask, add.x);
    }
}

// The score of a decision after a binding cap vertex.
__device__ __forceinline__ void score(Prb &G, uint32_t param, float dlog_p) {
    if (G.binding && G.after_capture() && param != kNoParam) G.sink.add(param, G.score * dlog_p);
}

// d log(ring_bsdf) / d tau, differentiating the piecewise forms of
// rings.wgsl:143-166 exactly as ring_bsdf evaluates them.
__device__ __forceinline__ float ring_bsdf_dlog_tau(float tau, float outgoing, float incoming) {
    if (!(tau > 0.0f)) return 0.0f;
    const float mo = fmaxf(fabsf(outgoing), 1.0e-7f);
    const float mi = fmaxf(fabsf(incoming), 1.0e-7f);
    if (outgoing * incoming < 0.0f) {
        // tau / (mo mi) * exp(-tau min(1/mo, 1/mi)) * integral(delta),
        // delta = tau |1/mo - 1/mi|.
        const float k = fabsf(1.0f / mo - 1.0f / mi);
        const float delta = fabsf(tau / mo - tau / mi);
        float dlog_integral;
        if (delta < 1.0e-3f) dlog_integral = -0.5f / (1.0f - 0.5f * delta);
        else if (delta < 0.05f) dlog_integral = -0.5f + delta / 12.0f - delta * delta * delta / 720.0f;
        else dlog_integral = 1.0f / expm1f(delta) - 1.0f / delta;
        return 1.0f / tau - fminf(1.0f / mo, 1.0f / mi) + k * dlog_integral;
    }
    // one_minus_exp(tau (1/mo + 1/mi)) / (mo + mi)
    const float k = 1.0f / mo + 1.0f / mi;
    const float x = tau / mo + tau / mi;
    if (x < 1.0e-3f) return 1.0f / tau - 0.5f * k / (1.0f - 0.5f * x);
    return k / expm1f(x);
}

// The table parameter behind a ring point (kNoParam when the ring has no
// tabulated profile); `scale` is d tau / d table value (ring_params.y).
__device__ __forceinline__ uint32_t tau_param(const Scene &S, uint32_t body, float3 point, float *scale) {
    const float4 params = bf(S, body, kRingParams);
    if (params.w < 0.5f) return kNoParam;
    const uint32_t slot = (uint32_t)params.w - 1u;
    const uint32_t bins = slot < SG_RING_TABLE_SLOTS ? S.p->bins[slot] : 0u;
    if (bins == 0u) return kNoParam;
    *scale = params.y;
    return slot * SG_RING_TABLE_MAX_BINS + ring_bin(ring_x(S, body, point), bins);
}

// d log scatter_probability / d table value: one_minus_exp(tau / |mu|)
// (rings.wgsl:143-145, pathtrace.wgsl:1423-1425) with tau = scale * table.
__device__ __forceinline__ float scatter_pdf_dlog(float tau, float mu_out, float scale) {
    const float m = fmaxf(fabsf(mu_out), 1.0e-7f);
    const float x = tau / m;
    const float p = one_minus_exp(x);
    if (!(p > 0.0f)) return 0.0f;
    return (x < 1.0e-3f ? 1.0f - x : expf(-x)) * (scale / m) / p;
}


// A crossing multiplies by exp(-tau / |mu|) (rings.wgsl:83-86):
// d log / d table = -scale / |mu|.
__device__ __forceinline__ GradEntry crossing_entry(const Scene &S, uint32_t body, float3 point, float3 d) {
    float scale = 0.0f;
    const uint32_t tp = tau_param(S, body, point, &scale);
    if (tp == kNoParam) return no_entry();
    const float mu = fmaxf(fabsf(dot_rn(d, xyz(bf(S, body, kRingPlane)))), 1.0e-7f);
    return scalar_entry(tp, -scale / mu);
}

// light_visibility (rings.wgsl:90-115) that also returns the ring crossings
// behind its transmission as derivative entries, for the adjoint.
struct Visibility {
    float v;
    uint32_t n;
    GradEntry cross[kMaxCrossings];
};

template <bool C, bool L, bool F>
static __device__ SG_ADJ_HOOK Visibility light_visibility_grad(Scene S, Counter<C, L, F> K, Ray r, uint32_t light,
                                                         bool entries) {
    Crossings rec;
    rec.n = 0;
    Visibility out;
    out.v = visibility_core(S, K, r, light, &rec);
    out.n = 0;
    if (out.v <= 0.0f || !entries) return out;
#pragma unroll
    for (int k = 0; k < kMaxCrossings; ++k) {
        if ((uint32_t)k >= rec.n) break;
        const GradEntry e = crossing_entry(S, rec.body[k], rec.point[k], r.d);
        if (e.param != kNoParam) out.cross[out.n++] = e;
    }
    // Crossings beyond the record are counted as dropped.
    if (rec.n > (uint32_t)kMaxCrossings) out.n += rec.n - (uint32_t)kMaxCrossings;
    return out;
}

__device__ __forceinline__ void crossing_factors(Prb &G, const Visibility &vis) {
#pragma unroll
    for (int k = 0; k < kMaxCrossings; ++k)
        if ((uint32_t)k < vis.n) G.local_factor(vis.cross[k]);
    if (vis.n > (uint32_t)kMaxCrossings) G.dropped += vis.n - (uint32_t)kMaxCrossings;
}

// The adjoint's view of a ring vertex: its table parameter, d tau / d
// table value, and d log of the vertex's scatter pdf.
struct RingVertexGrad {
    uint32_t param;
    float scale;
    float dlog_pdf;
};

static __device__ SG_ADJ_HOOK RingVertexGrad ring_vertex_grad(Scene S, uint32_t ring, float3 point, float tau,
                                                        float mu_out) {
    RingVertexGrad v{kNoParam, 0.0f, 0.0f};
    v.param = tau_param(S, ring, point, &v.scale);
    if (v.param != kNoParam) v.dlog_pdf = scatter_pdf_dlog(tau, mu_out, v.scale);
    return v;
}

// The slab BSDF's optical-depth entry at a ring vertex for an incoming
// cosine.
__device__ __forceinline__ GradEntry ring_tau_entry(const RingVertexGrad &v, float tau, float outgoing,
                                                    float incoming) {
    return v.param == kNoParam ? no_entry() : scalar_entry(v.param, v.scale * ring_bsdf_dlog_tau(tau, outgoing, incoming));
}

// One light sample at a ring vertex (pathtrace.wgsl:1437-1450): its
// radiance, and at the cap vertex of a binding path its term of the cap
// (max(shadowed, 0.003 * unshadowed) luminance of `lit`). After the cap
// vertex the MIS weight's dependence on the vertex's scatter pdf is an
// attached entry.
static __device__ SG_ADJ_HOOK void ring_light_grad(Scene S, Prb &G, uint32_t ring, Optics optics, float mu_out,
                                             float mu_in, uint32_t light, float3 lit, Visibility vis, float weight,
                                             float ring_mis, bool last_vertex, RingVertexGrad vg) {
    const GradEntry tau_e = ring_tau_entry(vg, optics.tau, mu_out, mu_in);
    const GradEntry albedo_e = ring_albedo_entry(G, ring);
    const GradEntry light_e = emitter_entry(G, light);
    const float3 value = lit * (vis.v * weight * ring_mis);
    if (value.x != 0.0f || value.y != 0.0f || value.z != 0.0f) {
        G.local_factor(tau_e);
        G.local_factor(albedo_e);
        G.local_factor(light_e);
        crossing_factors(G, vis);
        if (G.post() && G.binding && !last_vertex && vg.param != kNoParam)
            G.local_factor(scalar_entry(vg.param | kPdfBit, -2.0f * (1.0f - weight) * vg.dlog_pdf));
        contribute(G, value, false);
    }
    if (G.binding && G.iteration == G.capture_iter) {
        const float3 cap_value = G.cap_direct ? lit * vis.v : lit * kRingIndirectCap;
        if (cap_value.x != 0.0f || cap_value.y != 0.0f || cap_value.z != 0.0f) {
            G.local_factor(tau_e);
            G.local_factor(albedo_e);
            G.local_factor(light_e);
            if (G.cap_direct) crossing_factors(G, vis);
            contribute(G, cap_value, true);
        }
    }
}

// A null crossing (pathtrace.wgsl:1451-1456): the transmission factor, and
// after a binding cap vertex the decision's score d log T.
static __device__ SG_ADJ_HOOK void ring_null_grad(Scene S, Prb &G, uint32_t ring, float3 point, float3 d) {
    const GradEntry ce = crossing_entry(S, ring, point, d);
    factor(G, ce);
    score(G, ce.param, ce.dlog.x);
}

// A ring scatter (pathtrace.wgsl:1466-1483): the slab BSDF's factors; after
// a binding cap vertex also the decision's score d log(1 - T) and the
// attached 1 / scatter pdf. Records the vertex for the MIS weight of an
// emitter reached next.
static __device__ SG_ADJ_HOOK void ring_scatter_grad(Scene S, Prb &G, uint32_t ring, Optics optics, float mu_out,
                                               float z, RingVertexGrad v, float transmission, float3 d) {
    factor(G, ring_tau_entry(v, optics.tau, mu_out, z));
    factor(G, ring_albedo_entry(G, ring));
    if (G.binding && v.param != kNoParam) {
        const float dlog_t = -v.scale / fmaxf(fabsf(dot_rn(d, xyz(bf(S, ring, kRingPlane)))), 1.0e-7f);
        if (transmission < 1.0f) score(G, v.param, -dlog_t * transmission / (1.0f - transmission));
        factor(G, scalar_entry(v.param | kPdfBit, -v.dlog_pdf));
    }
    G.prev_param = v.param;
    G.prev_dlog_pdf = v.dlog_pdf;
}

// One light sample at a surface vertex (pathtrace.wgsl:1545-1565).
static __device__ SG_ADJ_HOOK void surface_light_grad(Prb &G, GradEntry albedo_e, uint32_t light, float3 value,
                                                Visibility vis) {
    G.local_factor(albedo_e);
    G.local_factor(emitter_entry(G, light));
    crossing_factors(G, vis);
    contribute(G, value, false);
}

// An emitter reached by the path (pathtrace.wgsl:1516-1526); `mis` is the
// MIS weight against the previous vertex's light sample, whose bsdf pdf
// (a ring scatter's) moves with that vertex's optical depth.
static __device__ SG_ADJ_HOOK void emitter_grad(Prb &G, uint32_t body, float3 value, float mis, bool weighted) {
    G.local_factor(emitter_entry(G, body));
    if (G.binding && G.post() && weighted && G.prev_param != kNoParam)
        G.local_factor(scalar_entry(G.prev_param | kPdfBit, 2.0f * (1.0f - mis) * G.prev_dlog_pdf));
    contribute(G, value, false);
}

// The albedo entry of a surface vertex: body colour of a celestial surface
// (zero where the clamp of surface_albedo is active), or the albedo-map
// texel of the host ground.
template <bool L>
static __device__ SG_ADJ_HOOK GradEntry albedo_entry(Scene S, const float4 *inv, Ray ray, float t, uint32_t index,
                                               float3 albedo) {
    if (index < kLocalBase) {
        const float4 m = inv[2u * index];
        const float3 d = f3(albedo.x > 0.0f && albedo.x < 1.0f ? m.x : 0.0f,
                            albedo.y > 0.0f && albedo.y < 1.0f ? m.y : 0.0f,
                            albedo.z > 0.0f && albedo.z < 1.0f ? m.z : 0.0f);
        return vector_entry(body_color_param(index), d);
    }
    if constexpr (L) {
        if ((index == kLocalBase || index == kTerrainId) && S.p->albedo_map) {
            const uint32_t texel = map_texel(S.p, landscape_point(S, ray, t));
            return scalar_entry(kGradMap + texel, inv_or_zero(S.p->albedo_map[texel]));
        }
    }
    return no_entry();
}

// ringshine with derivatives (pathtrace.wgsl:1248-1296): the same draws and
// result as ringshine(), plus one contribution per light. `carried` is the
// path throughput times the surface albedo.
template <bool C, bool L, bool F>
static __device__ SG_ADJ_HOOK Shine ringshine_grad(Scene S, Counter<C, L, F> K, uint32_t index, float3 origin, float3 normal,
                                             bool last_vertex, uint32_t rng, Prb &G, float3 carried,
                                             GradEntry albedo_e) {
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    if (!has_ring(S, index)) return Shine{zero, rng};
    const ShinePoint sp = shine_point(S, K, index, origin, normal, last_vertex, rng);
    rng = sp.rng;
    if (!sp.valid) return Shine{zero, rng};
    const float3 n = xyz(bf(S, index, kRingPlane));
    float scale = 0.0f;
    const uint32_t tp = tau_param(S, index, sp.point, &scale);
    const RingVertexGrad vg{tp, scale, 0.0f};
    float3 shine = zero;
    const uint32_t count = light_count(S.s);
#pragma unroll 1
    for (uint32_t slot = 0; slot < count; ++slot) {
        const uint32_t i = light_index(S.s, slot);
        const float4 material = bf(S, i, kMaterial);
        if (material.w < 0.5f) continue;
        const LightSample light = sample_light(S, K, Ray{sp.point, n, index}, i, rng);
        rng = light.rng;
        const float mu_in = dot(light.d, n);
        const Visibility vis = light_visibility_grad(S, K, ring_origin(S, index, sp.point, light.d), i, true);
        const float3 term = ring_bsdf(sp.optics, sp.mu_out, mu_in) * xyz(material) * (fabsf(mu_in) * vis.v / light.pdf);
        shine = shine + term;
        if (vis.v > 0.0f) {
            G.local_factor(albedo_e);
            G.local_factor(ring_tau_entry(vg, sp.optics.tau, sp.mu_out, mu_in));
            G.local_factor(ring_albedo_entry(G, index));
            G.local_factor(emitter_entry(G, i));
            crossing_factors(G, vis);
            contribute(G, carried * term * sp.scale, false);
        }
    }
    return Shine{shine * sp.scale, rng};
}

// Pass 1 hooks.
__device__ __forceinline__ void record_capture(Prb &G, uint32_t iteration, float cap, bool cap_direct, float3 base) {
    G.capture_iter = iteration;
    G.cap = cap;
    G.cap_direct = cap_direct;
    G.base = base;
    G.cap_light = cap_direct ? G.lit_vis_sum : G.lit_sum * kRingIndirectCap;
}

static __device__ SG_ADJ_HOOK void record_roulette(Prb &G, uint32_t iteration, float3 t, float s, bool survived,
                                             float3 radiance) {
    if (G.capture_iter == 0u) return;
    if (G.n_rr >= (uint32_t)kMaxRoulette) {
        G.dropped += 1u;
        return;
    }
    const float mx = fmaxf(t.x, fmaxf(t.y, t.z));
    const uint32_t m = t.x >= mx ? 0u : (t.y >= mx ? 1u : 2u);
    const bool clamped = !(mx > 0.05f && mx < 0.95f);
    const float3 before = radiance - G.base;
    const uint32_t bits = m | (survived ? 4u : 0u) | (clamped ? 8u : 0u);
    G.lists->rr[G.n_rr][0] = make_float4(__uint_as_float(iteration), __uint_as_float(bits), s, 0.0f);
    G.lists->rr[G.n_rr][1] = make_float4(before.x, before.y, before.z, 0.0f);
    G.n_rr += 1u;
}

// Start of pass 1 for a pixel weight w.
__device__ __forceinline__ void pass1_setup(Prb &G, float3 w) {
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    G.pass2 = false;
    G.known_total = false;
    G.capture_iter = 0;
    G.n_rr = 0;
    G.binding = false;
    G.iteration = 0;
    G.w_pre = w;
    G.w_post = w;
    G.w_pdf = zero;
    G.w_cap = zero;
    G.score = 0.0f;
    G.a = zero;
    G.b = zero;
    G.prev_param = kNoParam;
    G.prev_dlog_pdf = 0.0f;
    G.n_local = 0;
    G.n_fac = 0;
    G.deferral_full = false;
}

// Whether the ring-indirect cap binds on a path that pass 1 finished with
// radiance `total` (before the clamp).
__device__ __forceinline__ bool cap_binds(const Prb &G, float3 total) {
    return G.capture_iter != 0u && luminance(total - G.base) > G.cap;
}

// End of a path that pass 1 finished alone: each deferred factor's share of
// the weighted radiance gathered after it.
static __device__ SG_ADJ_HOOK void flush_deferred(Prb &G) {
#pragma unroll 1
    for (uint32_t k = 0; k < G.n_fac; ++k) {
        const GradEntry e = unpack_entry(G.lists->fac[k][0]);
        const float3 rem = G.a - xyz(G.lists->fac[k][1]);
        if (e.param & kVectorBit) {
            const uint32_t base = e.param & ~kVectorBit;
            G.sink.add(base + 0u, rem.x * e.dlog.x);
            G.sink.add(base + 1u, rem.y * e.dlog.y);
            G.sink.add(base + 2u, rem.z * e.dlog.z);
        } else {
            G.sink.add(e.param & kParamMask, sum3(rem) * e.dlog.x);
        }
    }
}

// Pass 2's weights from pass 1's summary, the path's total radiance and the
// pixel weight w.
static __device__ SG_ADJ_HOOK void pass2_setup(Prb &G, float3 total, float3 w) {
    const float3 lum = f3(0.2126f, 0.7152f, 0.0722f);
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    G.pass2 = true;
    G.known_total = false;
    G.w_pre = w;
    G.w_post = w;
    G.w_pdf = zero;
    G.w_cap = zero;
    G.score = 0.0f;
    G.a = zero;
    G.b = zero;
    G.b_total = zero;
    G.binding = false;
    G.prev_param = kNoParam;
    G.prev_dlog_pdf = 0.0f;
    G.iteration = 0;
    G.n_local = 0;
    if (G.capture_iter == 0u) {
        G.a_total = mul3(w, total);
        return;
    }
    const float3 indirect = total - G.base;
    const float l = luminance(indirect);
    if (l > G.cap) {
        const float s = G.cap / l;
        const float wc = dot(w, indirect) / l;
        G.binding = true;
        G.w_post = (w - lum * wc) * s;
        G.w_pdf = G.w_post - w;
        G.w_cap = lum * wc;
        G.score = (s - 1.0f) * dot(w, indirect);
        G.b_total = mul3(G.w_pdf, indirect);
        for (uint32_t r = 0; r < G.n_rr && r < (uint32_t)kMaxRoulette; ++r) {
            const float4 head = G.lists->rr[r][0];
            const float3 before = xyz(G.lists->rr[r][1]);
            const bool survived = (__float_as_uint(head.y) & 4u) != 0u;
            const float sr = head.z;
            G.lists->rr[r][0].w = survived ? G.score - dot(G.w_pdf, indirect - before) : -G.score * sr / (1.0f - sr);
        }
    } else {
        G.n_rr = 0;
    }
    G.a_total = mul3(w, G.base) + mul3(G.w_post, indirect) + mul3(G.w_cap, G.cap_light);
}

// A segment of a checkpointed path whose ring-indirect cap does not bind:
// the path's radiance `total` (from the forward) and the radiance it had
// gathered at the segment's start `so_far` give every weight, so the
// segment replays once, from its checkpoint, with nothing deferred.
__device__ __forceinline__ void segment_setup(Prb &G, float3 w, float3 total, float3 so_far) {
    const float3 zero = f3(0.0f, 0.0f, 0.0f);
    G.pass2 = true;
    G.known_total = true;
    G.capture_iter = 0;
    G.n_rr = 0;
    G.binding = false;
    G.iteration = 0;
    G.w_pre = w;
    G.w_post = w;
    G.w_pdf = zero;
    G.w_cap = zero;
    G.score = 0.0f;
    G.a = mul3(w, so_far);
    G.b = zero;
    G.a_total = mul3(w, total);
    G.b_total = zero;
    G.prev_param = kNoParam;
    G.prev_dlog_pdf = 0.0f;
    G.n_local = 0;
    G.n_fac = 0;
    G.deferral_full = false;
}

}  // namespace sg
