// sg_host.cpp — C-ABI host runtime of the B200 integrator.
//
// Mirrors the host side of stargaze's `PathTracer` (src/pathtracer.rs):
// options and their defaults (:77-111), the sample History and its reset key
// (:164-188), quality control (:761-773), and `encode` (:789-1009): capacity
// checks, batch clamping, Settings packing and the trace dispatch. wgpu
// buffers become device allocations owned by the context; `assert!` panics
// become SG_ERR_* status codes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "../../include/stargaze_b200.h"
#include "sg_internal.h"

namespace {

// sky::WIDTH / sky::HEIGHT (Milky Way map size, src/sky.rs) and
// stars::POINT_SOURCE_GAIN (src/stars.rs:130), as packed into
// Settings.background by encode (src/pathtracer.rs:853-858).
constexpr float kMilkyWayWidth = 1024.0f;
constexpr float kMilkyWayHeight = 512.0f;
constexpr float kPointSourceGain = 100.0f;
// Default terrain grid of the forest ground (src/terrain.rs:10), packed as
// log2(cells) into ground_counts.z bits 8..15 (src/pathtracer.rs:825-828).
constexpr uint32_t kDefaultTerrainCells = 512;

thread_local std::string g_last_error;

struct History {
    std::vector<uint8_t> key;
    uint64_t key_hash = 0;
    uint32_t samples = 0;
    uint32_t sequence = 0;
    // Noise-key runs (first key, count) of the samples behind the
    // accumulation, for the adjoint's replay; `replayable` false once the
    // accumulation was restored from outside or the runs overflowed.
    std::vector<std::pair<uint32_t, uint32_t>> runs;
    bool replayable = true;
};

}  // namespace

struct sg_context {
    int device = 0;
    uint32_t width = 0, height = 0;
    sg_options options{};
    History history;
    uint32_t exposure_idle_frames = 0;
    float4 *mean = nullptr;
    float4 *sum = nullptr;
    float4 *comp = nullptr;
    float4 *backdrop = nullptr;
    sg_sphere *bodies = nullptr;  // SG_BODY_CAPACITY
    float *ring_tables = nullptr; // SG_RING_TABLE_SLOTS * SG_RING_TABLE_MAX_BINS
    uint32_t ring_bins[SG_RING_TABLE_SLOTS] = {};
    uint64_t table_version = 0;
    unsigned long long *events = nullptr;  // kEventCount counters
    void *scratch = nullptr;               // query staging
    size_t scratch_bytes = 0;
    uint64_t launches = 0;
    std::string last_error;
    // Local landscape.
    sg_primitive *props = nullptr;  // SG_PROP_CAPACITY
    float4 *prop_trig = nullptr;    // 2 float4 per prop
    std::vector<float4> trig_host;
    float *terrain = nullptr;       // full layout incl. the geometry cache
    uint32_t terrain_cells = 0;
    uint32_t terrain_detail = 0;            // floats of the basalt elevation atlas
    bool terrain_cached = false;
    float terrain_radius = 0.0f;    // host radius the cache was built for
    float *albedo_map = nullptr;
    uint32_t map_width = 0, map_height = 0;
    float map_extent = 0.0f;
    bool fp64_sites = false;                // ring plane, host sphere, 5 mm offset in FP64
    bool guided_ground = false;             // the guided ground sampler (air frames)
    bool ringshine = true;                  // ringshine NEE at ringed bodies' surfaces
    // Wavefront integrator (sg_set_integrator), buffers allocated on first use.
    int integrator = SG_INTEGRATOR_WAVEFRONT;
    uint32_t wave_pool_request = 0;         // 0: the default pool
    float4 *wave_state = nullptr;           // planes, hit planes, queues, counters
    size_t wave_state_size = 0;
    uint32_t wave_pool = 0;
    float4 *wave_results = nullptr;         // per-sample radiance + running totals
    void *adjoint_slots = nullptr;          // staged adjoint: slot state, lists, free ring
    size_t adjoint_slots_size = 0;
    size_t wave_results_size = 0;
    sg::WaveProgress wave_progress;         // the stage loops' progress ring (mapped host memory)
    uint32_t wave_iterations = 0;           // stage iterations of the last dispatch
    // Sky backdrop: catalogue (2 float4 per star), cell table, panorama.
    float4 *catalogue = nullptr;
    uint32_t catalogue_n = 0;
    uint32_t *sky_cells = nullptr;
    uint32_t *milky_way = nullptr;
    uint32_t milky_width = 0, milky_height = 0;
    float4 *sky_samples = nullptr;          // wavefront: per-sample backdrop + totals
    size_t sky_samples_size = 0;
    bool backdrop_written = false;          // the backdrop buffer holds a sky
    // Host air: the surface sky cache (128 float4), rebuilt when an
    // accumulation starts.
    float4 *sky_light = nullptr;
    // Display: the exposure state and histogram of the metering.
    sg::ExposureState *exposure = nullptr;
    uint32_t *histogram = nullptr;
    bool exposure_was_enabled = false;
    bool stage_timing = false;              // bracket every stage with events
    sg::StageMarks stage_marks;
    float stage_ms[sg::kStageCount] = {};   // per stage, last timed dispatch
    // Adjoint buffers, allocated on first use.
    float *grad = nullptr;                  // kGradMap + texels floats
    size_t grad_floats = 0;
    float4 *dl_dimage = nullptr;            // staging of a host d loss / d image
    size_t dl_pixels = 0;
    unsigned long long *dropped = nullptr;  // one counter
    // Vertex checkpoints (sg_set_checkpoints): settings, then the buffers of
    // the current accumulation.
    uint32_t ck_every = 0;
    uint32_t ck_samples = 0;                // accumulation samples covered
    uint64_t ck_record_bytes = 0;           // record budget (0: automatic)
    float4 *ck_records = nullptr;
    uint32_t ck_capacity = 0;
    float4 *ck_totals = nullptr;
    size_t ck_totals_size = 0;
    uint32_t *ck_count = nullptr;
    bool ck_valid = false;                  // every sample so far went through the checkpointing forward
    uint2 *camera_cull = nullptr;           // per-tile cull masks of camera rays
    size_t camera_cull_tiles = 0;
};

namespace {

int fail(sg_context *ctx, int status, const std::string &message) {
    if (ctx) ctx->last_error = message;
    g_last_error = message;
    return status;
}

int cuda_fail(sg_context *ctx, cudaError_t e, const char *what) {
    std::string msg = std::string(what) + ": " + cudaGetErrorString(e);
    return fail(ctx, e == cudaErrorMemoryAllocation ? SG_ERR_OOM : SG_ERR_CUDA, msg);
}

#define SG_CUDA(ctx, call)                                   \
    do {                                                     \
        cudaError_t _e = (call);                             \
        if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
    } while (0)

struct DeviceGuard {
    int previous = -1;
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&previous) != cudaSuccess) previous = -1;
        if (previous != device) cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (previous >= 0) cudaSetDevice(previous);
    }
};

void free_image(sg_context *ctx) {
    cudaFree(ctx->mean);
    cudaFree(ctx->sum);
    cudaFree(ctx->comp);
    cudaFree(ctx->backdrop);
    ctx->mean = ctx->sum = ctx->comp = ctx->backdrop = nullptr;
}

int alloc_image(sg_context *ctx) {
    // accumulation() in src/pathtracer.rs:277-289 sizes at least 16 bytes.
    const size_t pixels = std::max<size_t>((size_t)ctx->width * ctx->height, 1);
    const size_t bytes = pixels * sizeof(float4);
    SG_CUDA(ctx, cudaMalloc(&ctx->mean, bytes));
    SG_CUDA(ctx, cudaMalloc(&ctx->sum, bytes));
    SG_CUDA(ctx, cudaMalloc(&ctx->comp, bytes));
    SG_CUDA(ctx, cudaMalloc(&ctx->backdrop, bytes));
    SG_CUDA(ctx, cudaMemset(ctx->mean, 0, bytes));
    SG_CUDA(ctx, cudaMemset(ctx->sum, 0, bytes));
    SG_CUDA(ctx, cudaMemset(ctx->comp, 0, bytes));
    SG_CUDA(ctx, cudaMemset(ctx->backdrop, 0, bytes));
    return SG_OK;
}

void reset_history(sg_context *ctx) {
    const uint32_t sequence = ctx->history.sequence;
    ctx->history = History{};
    ctx->history.sequence = sequence;
}

template <typename T>
void append(std::vector<uint8_t> &key, const T &value) {
    const uint8_t *p = reinterpret_cast<const uint8_t *>(&value);
    key.insert(key.end(), p, p + sizeof(T));
}

// FNV-1a over the history key: the tape's check that a backward replays
// the frame its samples were rendered with.
uint64_t key_hash(const std::vector<uint8_t> &key) {
    uint64_t h = 1469598103934665603ull;
    for (uint8_t b : key) h = (h ^ b) * 1099511628211ull;
    return h;
}

// History::update (src/pathtracer.rs:173-187): the accumulation survives
// only while globals, bodies, ground, scene time, bounces, Milky Way
// brightness (and here the ring tables) are byte-identical.
std::vector<uint8_t> history_key(const sg_context *ctx, const sg_frame *frame) {
    std::vector<uint8_t> key;
    key.reserve(sizeof(sg_globals) + frame->n_bodies * sizeof(sg_sphere) + frame->n_ground * sizeof(sg_primitive) + 32);
    append(key, *frame->globals);
    if (frame->n_bodies)
        key.insert(key.end(), reinterpret_cast<const uint8_t *>(frame->bodies),
                   reinterpret_cast<const uint8_t *>(frame->bodies + frame->n_bodies));
    if (frame->n_ground)
        key.insert(key.end(), reinterpret_cast<const uint8_t *>(frame->ground),
                   reinterpret_cast<const uint8_t *>(frame->ground + frame->n_ground));
    append(key, frame->scene_time);
    append(key, ctx->options.max_bounces);
    append(key, ctx->options.milky_way);
    append(key, ctx->table_version);
    append(key, ctx->fp64_sites);
    append(key, ctx->guided_ground);
    append(key, ctx->ringshine);
    append(key, ctx->ck_every);
    return key;
}

void update_history(sg_context *ctx, const sg_frame *frame) {
    std::vector<uint8_t> key = history_key(ctx, frame);
    if (key != ctx->history.key) {
        ctx->history.key_hash = key_hash(key);
        ctx->history.key = std::move(key);
        ctx->history.samples = 0;
        ctx->history.runs.clear();
        ctx->history.replayable = true;
    }
}

// Record a dispatch's noise keys [first, first + count) for the tape.
void record_run(sg_context *ctx, uint32_t first, uint32_t count) {
    auto &runs = ctx->history.runs;
    if (!runs.empty() && runs.back().first + runs.back().second == first) {
        runs.back().second += count;
    } else if (runs.size() < SG_TAPE_RANGES) {
        runs.emplace_back(first, count);
    } else {
        ctx->history.replayable = false;
    }
}

// Validation shared by encode and the probes (src/pathtracer.rs:795-800
// plus the features this build does not implement yet).
int validate_frame(sg_context *ctx, const sg_frame *frame) {
    if (!frame || !frame->globals) return fail(ctx, SG_ERR_INVALID, "frame or frame->globals is NULL");
    if (frame->n_bodies > SG_BODY_CAPACITY) return fail(ctx, SG_ERR_CAPACITY, "too many scene bodies");
    if (frame->n_bodies && !frame->bodies) return fail(ctx, SG_ERR_INVALID, "frame->bodies is NULL");
    if (frame->n_ground > SG_PROP_CAPACITY) return fail(ctx, SG_ERR_CAPACITY, "too many local primitives");
    if (frame->n_ground && !frame->ground) return fail(ctx, SG_ERR_INVALID, "frame->ground is NULL");
    if (frame->globals->ground_counts[0] != frame->n_ground)
        return fail(ctx, SG_ERR_INVALID, "ground_counts.x does not match the primitive count");
    const float host = frame->globals->ground_north[3];
    if (host != 0.0f) {
        if (host != std::floor(host) || host < 1.0f || host > (float)frame->n_bodies)
            return fail(ctx, SG_ERR_INVALID, "ground_north.w must be 0 or a body index + 1");
        if ((frame->globals->ground_counts[2] & 255u) > 5u)
            return fail(ctx, SG_ERR_INVALID, "landscape themes above 5 do not exist");
        if (frame->globals->ground_counts[1] != 0u && !ctx->terrain)
            return fail(ctx, SG_ERR_STATE, "terrain is enabled but no terrain was uploaded");
        if (!(frame->globals->ground_up[3] > 0.0f))
            return fail(ctx, SG_ERR_INVALID, "ground_up.w (host radius in metres) must be positive");
        for (uint32_t i = 0; i < frame->n_ground; ++i) {
            const float kind = frame->ground[i].center[3];
            if (kind < 0.0f && (kind != std::floor(kind) || (double)i - (double)kind >= (double)frame->n_ground + 1.0))
                return fail(ctx, SG_ERR_INVALID, "a group marker skips past the end of the primitive list");
        }
    }
    for (uint32_t i = 0; i < frame->n_bodies; ++i) {
        const float slot = frame->bodies[i].ring_params[3];
        if (slot >= 0.5f && (slot > (float)SG_RING_TABLE_SLOTS || slot != std::floor(slot)))
            return fail(ctx, SG_ERR_INVALID, "ring_params.w must be 0 or a ring-table slot + 1");
    }
    return SG_OK;
}

// The Settings packing of encode (src/pathtracer.rs:812-859).
sg_settings pack_settings(const sg_context *ctx, const sg_frame *frame, uint32_t count) {
    sg_settings s;
    std::memset(&s, 0, sizeof(s));
    s.g = *frame->globals;
    s.g.viewport[3] = s.g.viewport[0] / std::max(s.g.viewport[1], 1.0f);
    s.g.viewport[0] = (float)ctx->width;
    s.g.viewport[1] = (float)ctx->height;
    s.g.viewport[2] = ctx->options.exposure;
    float prop_top = 0.0f;
    for (uint32_t i = 0; i < frame->n_ground; ++i) {
        const float *e = frame->ground[i].extent;
        const float len = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
        prop_top = std::max(prop_top, frame->ground[i].center[1] + len);
    }
    std::memcpy(&s.g.ground_counts[3], &prop_top, sizeof(float));
    uint32_t cells = ctx->terrain_cells ? ctx->terrain_cells : kDefaultTerrainCells, log2 = 0;
    while ((1u << log2) < cells) ++log2;
    // The reference ORs log2(cells) over the theme byte; stale grid bits in
    // the caller's frame are cleared first so they cannot name a grid that
    // was not uploaded.
    s.g.ground_counts[2] = (s.g.ground_counts[2] & 255u) | (log2 << 8);
    for (uint32_t i = 0; i < frame->n_bodies; ++i) {
        if (frame->bodies[i].emissive >= 0.5f) {
            if (s.lights[3] < 3u) s.lights[s.lights[3]] = i;
            s.lights[3] += 1u;
        }
    }
    s.sampling[0] = ctx->options.noise_seed + ctx->history.sequence;
    s.counts[0] = frame->n_bodies;
    s.counts[1] = ctx->history.samples;
    s.counts[2] = count;
    s.counts[3] = ctx->options.max_bounces;
    s.background[0] = ctx->options.milky_way;
    s.background[1] = ctx->milky_way ? (float)ctx->milky_width : kMilkyWayWidth;
    s.background[2] = ctx->milky_way ? (float)ctx->milky_height : kMilkyWayHeight;
    s.background[3] = kPointSourceGain;
    return s;
}

// Write the frame's bodies and landscape primitives (src/pathtracer.rs:
// 907-913) and refresh the terrain geometry cache when the host radius
// changed (:933-945).
int upload_bodies(sg_context *ctx, const sg_frame *frame, cudaStream_t stream) {
    if (frame->n_bodies)
        SG_CUDA(ctx, cudaMemcpyAsync(ctx->bodies, frame->bodies, frame->n_bodies * sizeof(sg_sphere),
                                     cudaMemcpyHostToDevice, stream));
    if (frame->globals->ground_north[3] == 0.0f) return SG_OK;
    if (frame->n_ground) {
        if (!ctx->props) SG_CUDA(ctx, cudaMalloc(&ctx->props, SG_PROP_CAPACITY * sizeof(sg_primitive)));
        if (!ctx->prop_trig) SG_CUDA(ctx, cudaMalloc(&ctx->prop_trig, SG_PROP_CAPACITY * 2 * sizeof(float4)));
        SG_CUDA(ctx, cudaMemcpyAsync(ctx->props, frame->ground, frame->n_ground * sizeof(sg_primitive),
                                     cudaMemcpyHostToDevice, stream));
        // Rotation sines and cosines per primitive (ground.wgsl:33-61): the
        // tumble angles of kind 2.25 (24 packed bits, TAU/256 steps) or the
        // yaw, each evaluated in double and rounded to f32 once per frame.
        ctx->trig_host.resize((size_t)frame->n_ground * 2);
        const float step = 6.283185307179586f / 256.0f;
        for (uint32_t i = 0; i < frame->n_ground; ++i) {
            const sg_primitive &p = frame->ground[i];
            float4 t0 = make_float4(0.0f, 1.0f, 0.0f, 1.0f), t1 = make_float4(0.0f, 1.0f, 0.0f, 0.0f);
            if (p.center[3] == 2.25f) {
                const uint32_t bits = (uint32_t)p.extent[3];
                const float ax = (float)(bits & 255u) * step, ay = (float)((bits >> 8) & 255u) * step;
                const float az = (float)((bits >> 16) & 255u) * step;
                t0 = make_float4((float)std::sin((double)ax), (float)std::cos((double)ax), (float)std::sin((double)ay),
                                 (float)std::cos((double)ay));
                t1 = make_float4((float)std::sin((double)az), (float)std::cos((double)az), 0.0f, 0.0f);
            } else if (p.center[3] >= 0.0f) {
                const double yaw = (double)p.extent[3];
                t1 = make_float4((float)std::sin(yaw), (float)std::cos(yaw), 0.0f, 0.0f);
            }
            ctx->trig_host[2 * i] = t0;
            ctx->trig_host[2 * i + 1] = t1;
        }
        SG_CUDA(ctx, cudaMemcpyAsync(ctx->prop_trig, ctx->trig_host.data(), ctx->trig_host.size() * sizeof(float4),
                                     cudaMemcpyHostToDevice, stream));
    }
    const float radius = frame->globals->ground_up[3];
    if (ctx->terrain && frame->globals->ground_counts[1] != 0u &&
        (!ctx->terrain_cached || ctx->terrain_radius != radius)) {
        cudaError_t e = sg::launch_terrain_cache(ctx->terrain, ctx->terrain_cells, radius, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "terrain cache launch");
        ctx->terrain_cached = true;
        ctx->terrain_radius = radius;
    }
    return SG_OK;
}

// Whether primary misses see a sky: a catalogue, or a panorama with a
// positive brightness.
bool sky_on(const sg_context *ctx) {
    return ctx->catalogue_n > 0u || (ctx->milky_way && ctx->options.milky_way > 0.0f);
}

sg::TraceParams make_params(sg_context *ctx, const sg_settings &s) {
    sg::TraceParams p;
    std::memset(&p, 0, sizeof(p));
    p.s = s;
    p.bodies = reinterpret_cast<const float4 *>(ctx->bodies);
    p.tables = ctx->ring_tables;
    uint32_t used_floats = 0;
    for (int k = 0; k < SG_RING_TABLE_SLOTS; ++k) {
        p.bins[k] = ctx->ring_bins[k];
        if (ctx->ring_bins[k]) used_floats = (uint32_t)(k + 1) * SG_RING_TABLE_MAX_BINS;
    }
    p.table_stride = SG_RING_TABLE_MAX_BINS;
    // Stage the tables in shared memory when the used slots fit in 32 KB.
    p.staged_table_floats = used_floats * sizeof(float) <= 32u * 1024u ? used_floats : 0u;
    p.mean = ctx->mean;
    p.sum = ctx->sum;
    p.comp = ctx->comp;
    p.width = ctx->width;
    p.height = ctx->height;
    p.events = nullptr;
    p.terrain = ctx->terrain;
    p.terrain_cells = ctx->terrain_cells;
    p.terrain_detail_floats = ctx->terrain_detail;
    p.props = reinterpret_cast<const float4 *>(ctx->props);
    p.prop_trig = ctx->prop_trig;
    p.n_props = s.g.ground_counts[0];
    p.albedo_map = ctx->albedo_map;
    p.map_width = ctx->map_width;
    p.map_height = ctx->map_height;
    p.map_extent = ctx->map_extent;
    p.fp64_sites = ctx->fp64_sites ? 1u : 0u;
    p.catalogue = ctx->catalogue;
    p.sky_cells = ctx->sky_cells;
    p.catalogue_n = ctx->catalogue_n;
    p.milky_way = ctx->milky_way;
    p.sky_on = sky_on(ctx) ? 1u : 0u;
    p.backdrop = ctx->backdrop;
    p.air_on = s.g.atmo_params[3] >= 0.5f ? 1u : 0u;
    p.sky_light = ctx->sky_light;
    p.guided_ground = ctx->guided_ground ? 1u : 0u;
    p.ringshine = ctx->ringshine ? 1u : 0u;
    return p;
}

// Options the integrator can run: the reference clamps bounces to 1..64
// (src/pathtracer.rs:114-122, :761-773); zero bounces would leave the path
// loop to Russian roulette alone.
int validate_options(sg_context *ctx, const sg_options *o) {
    if (o->max_bounces < 1u || o->max_bounces > 64u)
        return fail(ctx, SG_ERR_INVALID, "max_bounces must be in 1..64");
    if (!std::isfinite(o->milky_way) || o->milky_way < 0.0f)
        return fail(ctx, SG_ERR_INVALID, "milky_way must be finite and non-negative");
    return SG_OK;
}

int ensure_scratch(sg_context *ctx, size_t bytes) {
    if (ctx->scratch_bytes >= bytes) return SG_OK;
    cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    SG_CUDA(ctx, cudaMalloc(&ctx->scratch, bytes));
    ctx->scratch_bytes = bytes;
    return SG_OK;
}

}  // namespace

extern "C" {

int sg_default_options(sg_options *o) {
    if (!o) return SG_ERR_INVALID;
    o->noise_seed = 0;
    o->samples_per_frame = 1;
    o->max_bounces = 8;
    o->sample_limit = SG_MAX_SAMPLES;
    o->exposure = 1.0f;
    o->auto_exposure = 0;
    o->ev_bias = 0.0f;
    o->auto_key = 0.25f;
    o->auto_percentile = 0.9f;
    o->milky_way = 4.0e-4f;
    return SG_OK;
}

int sg_create(int device, uint32_t width, uint32_t height, const sg_options *options, sg_context **out) {
    if (!out) return fail(nullptr, SG_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return fail(nullptr, SG_ERR_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
    if (device < 0 || device >= count) return fail(nullptr, SG_ERR_INVALID, "no such CUDA device");
    if ((uint64_t)width * height > (1ull << 31)) return fail(nullptr, SG_ERR_INVALID, "viewport too large");
    if (options && validate_options(nullptr, options) != SG_OK) return SG_ERR_INVALID;
    sg_context *ctx = new (std::nothrow) sg_context();
    if (!ctx) return fail(nullptr, SG_ERR_OOM, "host allocation failed");
    ctx->device = device;
    ctx->width = width;
    ctx->height = height;
    if (options) ctx->options = *options;
    else sg_default_options(&ctx->options);
    DeviceGuard guard(device);
    int status = alloc_image(ctx);
    if (status == SG_OK) {
        if ((e = cudaMalloc(&ctx->bodies, SG_BODY_CAPACITY * sizeof(sg_sphere))) != cudaSuccess ||
            (e = cudaMalloc(&ctx->ring_tables, SG_RING_TABLE_SLOTS * SG_RING_TABLE_MAX_BINS * sizeof(float))) !=
                cudaSuccess ||
            (e = cudaMalloc(&ctx->events, sg::kEventCount * sizeof(unsigned long long))) != cudaSuccess)
            status = cuda_fail(ctx, e, "cudaMalloc");
    }
    if (status == SG_OK) {
        e = cudaMemset(ctx->ring_tables, 0, SG_RING_TABLE_SLOTS * SG_RING_TABLE_MAX_BINS * sizeof(float));
        if (e != cudaSuccess) status = cuda_fail(ctx, e, "cudaMemset");
    }
    if (status != SG_OK) {
        sg_destroy(ctx);
        return status;
    }
    *out = ctx;
    return SG_OK;
}

int sg_destroy(sg_context *ctx) {
    if (!ctx) return SG_OK;
    DeviceGuard guard(ctx->device);
    free_image(ctx);
    cudaFree(ctx->bodies);
    cudaFree(ctx->ring_tables);
    cudaFree(ctx->events);
    cudaFree(ctx->scratch);
    cudaFree(ctx->props);
    cudaFree(ctx->prop_trig);
    cudaFree(ctx->terrain);
    cudaFree(ctx->albedo_map);
    cudaFree(ctx->grad);
    cudaFree(ctx->dl_dimage);
    cudaFree(ctx->dropped);
    cudaFree(ctx->wave_state);
    cudaFree(ctx->wave_results);
    cudaFree(ctx->adjoint_slots);
    cudaFree(ctx->ck_records);
    cudaFree(ctx->ck_totals);
    cudaFree(ctx->ck_count);
    cudaFree(ctx->camera_cull);
    cudaFree(ctx->exposure);
    cudaFree(ctx->histogram);
    cudaFree(ctx->catalogue);
    cudaFree(ctx->sky_cells);
    cudaFree(ctx->milky_way);
    cudaFree(ctx->sky_samples);
    cudaFree(ctx->sky_light);
    if (ctx->wave_progress.host) cudaFreeHost(ctx->wave_progress.host);
    for (cudaEvent_t e : ctx->wave_progress.done)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : ctx->stage_marks.events) cudaEventDestroy(e);
    delete ctx;
    return SG_OK;
}

int sg_upload_terrain(sg_context *ctx, const float *data, size_t n_floats, uint32_t cells) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (cells < 2u || cells > SG_TERRAIN_MAX_CELLS || (cells & (cells - 1u)) != 0u)
        return fail(ctx, SG_ERR_INVALID, "cells must be a power of two in 2..4096");
    if (!data) return fail(ctx, SG_ERR_INVALID, "data is NULL");
    const size_t source = sg::terrain_source_floats(cells);
    // An optional tail after the source layout is the basalt elevation atlas
    // (src/volcano.rs), stored where volcano.wgsl reads it: after the cache.
    if (n_floats < source || n_floats - source > (size_t)UINT32_MAX)
        return fail(ctx, SG_ERR_INVALID, "terrain data length does not match the grid");
    const size_t detail = n_floats - source;
    const size_t full = sg::terrain_floats(cells);
    DeviceGuard guard(ctx->device);
    cudaDeviceSynchronize();
    cudaFree(ctx->terrain);
    ctx->terrain = nullptr;
    ctx->terrain_cells = 0;
    ctx->terrain_detail = 0;
    ctx->terrain_cached = false;
    SG_CUDA(ctx, cudaMalloc(&ctx->terrain, (full + detail) * sizeof(float)));
    SG_CUDA(ctx, cudaMemcpy(ctx->terrain, data, source * sizeof(float), cudaMemcpyHostToDevice));
    if (detail)
        SG_CUDA(ctx, cudaMemcpy(ctx->terrain + full, data + source, detail * sizeof(float), cudaMemcpyHostToDevice));
    ctx->terrain_cells = cells;
    ctx->terrain_detail = (uint32_t)detail;
    ctx->table_version += 1;
    return SG_OK;
}

int sg_upload_albedo_map(sg_context *ctx, const float *albedo, uint32_t width, uint32_t height, float extent_m) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    DeviceGuard guard(ctx->device);
    if (width == 0 || height == 0) {
        cudaDeviceSynchronize();
        cudaFree(ctx->albedo_map);
        ctx->albedo_map = nullptr;
        ctx->map_width = ctx->map_height = 0;
        ctx->table_version += 1;
        return SG_OK;
    }
    if (!albedo || !(extent_m > 0.0f) || (uint64_t)width * height > (1ull << 26))
        return fail(ctx, SG_ERR_INVALID, "albedo map needs data, a positive extent and at most 2^26 texels");
    for (size_t k = 0; k < (size_t)width * height; ++k)
        if (!(albedo[k] >= 0.0f && albedo[k] <= 1.0f))
            return fail(ctx, SG_ERR_INVALID, "albedo texels must lie in [0, 1]");
    cudaDeviceSynchronize();
    cudaFree(ctx->albedo_map);
    ctx->albedo_map = nullptr;
    SG_CUDA(ctx, cudaMalloc(&ctx->albedo_map, (size_t)width * height * sizeof(float)));
    SG_CUDA(ctx, cudaMemcpy(ctx->albedo_map, albedo, (size_t)width * height * sizeof(float), cudaMemcpyHostToDevice));
    ctx->map_width = width;
    ctx->map_height = height;
    ctx->map_extent = extent_m;
    ctx->table_version += 1;
    return SG_OK;
}

int sg_upload_catalogue(sg_context *ctx, const float *stars, uint32_t n, const uint32_t *cells, uint32_t n_cells) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    DeviceGuard guard(ctx->device);
    constexpr uint32_t kOffsets = 256u * 128u + 1u;
    if (n == 0) {
        cudaDeviceSynchronize();
        cudaFree(ctx->catalogue);
        cudaFree(ctx->sky_cells);
        ctx->catalogue = nullptr;
        ctx->sky_cells = nullptr;
        ctx->catalogue_n = 0;
        ctx->table_version += 1;
        return SG_OK;
    }
    if (!stars || !cells || n > (1u << 20) || n_cells < kOffsets)
        return fail(ctx, SG_ERR_INVALID, "catalogue needs 1..2^20 stars and a cell table of at least 32,769 words");
    if (cells[0] != 0u) return fail(ctx, SG_ERR_INVALID, "the first cell offset must be 0");
    for (uint32_t k = 1; k < kOffsets; ++k)
        if (cells[k] < cells[k - 1]) return fail(ctx, SG_ERR_INVALID, "cell offsets must not decrease");
    if (cells[kOffsets - 1] != n_cells - kOffsets)
        return fail(ctx, SG_ERR_INVALID, "the last cell offset must equal the number of indices");
    for (uint32_t k = kOffsets; k < n_cells; ++k)
        if (cells[k] >= n) return fail(ctx, SG_ERR_INVALID, "a cell lists a star beyond the catalogue");
    for (size_t k = 0; k < (size_t)n * 8u; ++k)
        if (!std::isfinite(stars[k])) return fail(ctx, SG_ERR_INVALID, "catalogue values must be finite");
    cudaDeviceSynchronize();
    cudaFree(ctx->catalogue);
    cudaFree(ctx->sky_cells);
    ctx->catalogue = nullptr;
    ctx->sky_cells = nullptr;
    ctx->catalogue_n = 0;
    SG_CUDA(ctx, cudaMalloc(&ctx->catalogue, (size_t)n * 2u * sizeof(float4)));
    SG_CUDA(ctx, cudaMalloc(&ctx->sky_cells, (size_t)n_cells * sizeof(uint32_t)));
    SG_CUDA(ctx, cudaMemcpy(ctx->catalogue, stars, (size_t)n * 2u * sizeof(float4), cudaMemcpyHostToDevice));
    SG_CUDA(ctx, cudaMemcpy(ctx->sky_cells, cells, (size_t)n_cells * sizeof(uint32_t), cudaMemcpyHostToDevice));
    ctx->catalogue_n = n;
    ctx->table_version += 1;
    return SG_OK;
}

int sg_upload_milky_way(sg_context *ctx, const uint32_t *texels, uint32_t width, uint32_t height) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    DeviceGuard guard(ctx->device);
    if (width == 0 || height == 0) {
        cudaDeviceSynchronize();
        cudaFree(ctx->milky_way);
        ctx->milky_way = nullptr;
        ctx->milky_width = ctx->milky_height = 0;
        ctx->table_version += 1;
        return SG_OK;
    }
    if (!texels || width > 16384 || height > 16384)
        return fail(ctx, SG_ERR_INVALID, "the panorama needs texels and at most 16384 x 16384 of them");
    for (size_t k = 0; k < (size_t)width * height; ++k)
        if (texels[k] >> 30) return fail(ctx, SG_ERR_INVALID, "panorama texels are 3 x 10-bit");
    cudaDeviceSynchronize();
    cudaFree(ctx->milky_way);
    ctx->milky_way = nullptr;
    SG_CUDA(ctx, cudaMalloc(&ctx->milky_way, (size_t)width * height * sizeof(uint32_t)));
    SG_CUDA(ctx, cudaMemcpy(ctx->milky_way, texels, (size_t)width * height * sizeof(uint32_t), cudaMemcpyHostToDevice));
    ctx->milky_width = width;
    ctx->milky_height = height;
    ctx->table_version += 1;
    return SG_OK;
}

int sg_resize(sg_context *ctx, uint32_t width, uint32_t height) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (width == ctx->width && height == ctx->height) return SG_OK;
    if ((uint64_t)width * height > (1ull << 31)) return fail(ctx, SG_ERR_INVALID, "viewport too large");
    DeviceGuard guard(ctx->device);
    cudaDeviceSynchronize();
    free_image(ctx);
    ctx->width = width;
    ctx->height = height;
    int status = alloc_image(ctx);
    if (status != SG_OK) return status;
    reset_history(ctx);
    ctx->exposure_idle_frames = 0;
    return SG_OK;
}

int sg_prepare_frame(sg_context *ctx, const sg_frame *frame, int *fresh) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    int status = validate_frame(ctx, frame);
    if (status != SG_OK) return status;
    update_history(ctx, frame);
    if (fresh) *fresh = ctx->history.samples == 0;
    return SG_OK;
}

int sg_set_quality(sg_context *ctx, uint32_t samples, uint32_t bounces, uint32_t limit) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    bounces = std::clamp<uint32_t>(bounces, 1u, 64u);
    if (ctx->options.max_bounces != bounces) {
        reset_history(ctx);
        ctx->exposure_idle_frames = 0;
    }
    ctx->options.samples_per_frame = std::clamp<uint32_t>(samples, 1u, 64u);
    ctx->options.max_bounces = bounces;
    ctx->options.sample_limit = std::clamp<uint32_t>(limit, 1u, SG_MAX_SAMPLES);
    return SG_OK;
}

int sg_set_options(sg_context *ctx, const sg_options *options) {
    if (!ctx || !options) return fail(ctx, SG_ERR_INVALID, "ctx or options is NULL");
    int status = validate_options(ctx, options);
    if (status != SG_OK) return status;
    ctx->options = *options;
    return SG_OK;
}

int sg_get_options(const sg_context *ctx, sg_options *options) {
    if (!ctx || !options) return SG_ERR_INVALID;
    *options = ctx->options;
    return SG_OK;
}

// Default pool of the wavefront integrator: 16 Mi paths (4.7 GB of state;
// smaller dispatches get a pool of their own size). On the 1080p ring
// workload 4, 8 and 16 Mi paths measured 6880, 7348 and 7649 Msamples/s:
// fewer, fuller iterations shorten the drain at the end of a dispatch.
constexpr uint32_t kDefaultWavePool = 1u << 24;
// Budget for the per-sample radiance the wavefront resolve sums in order:
// a 1080p dispatch of 64 samples fits in one chunk.
constexpr size_t kWaveResultBudget = (size_t)9 << 28;

// Default pool of the staged adjoint: 16 Mi paths (about 1.1 KB each with
// the adjoint slot, 17 GB), or the batch's sample count if smaller. On the
// ring scene (512^2, 64 spp) 4, 8 and 16 Mi paths measured 9.6, 9.1 and
// 8.7 ms; on the terrain scene (960x540, 64 spp) 59.7, 55.7 and 53.5 ms.
constexpr uint32_t kDefaultAdjointPool = 1u << 24;

// The pool for `samples` samples per pixel: the request (or `fallback`),
// at most the padded sample count, a multiple of 256.
static uint32_t wave_pool_for(const sg_context *ctx, uint32_t samples, uint32_t fallback) {
    const uint32_t tiles = ((ctx->width + 15u) / 16u) * ((ctx->height + 15u) / 16u);
    const uint64_t work = (uint64_t)tiles * 256u * samples;
    const uint32_t want = ctx->wave_pool_request ? ctx->wave_pool_request : fallback;
    return (uint32_t)std::min<uint64_t>(want, (work + 255u) & ~(uint64_t)255u);
}

// Whether the forward stores vertex records: some depth a scatter can reach
// (below the bounce limit) is a multiple of `every`.
static bool checkpoint_records(const sg_context *ctx) {
    return ctx->ck_every > 0u && ctx->ck_every < ctx->options.max_bounces;
}

// Path state planes, extend results, queues and counters for `pool` paths
// (the buffer grows only; forward and backward share it).
static int ensure_wave_state(sg_context *ctx, uint32_t pool, sg::WaveParams &w) {
    const size_t state_bytes = sg::wave_state_bytes(pool);
    if (state_bytes > ctx->wave_state_size) {
        cudaFree(ctx->wave_state);
        ctx->wave_state = nullptr;
        ctx->wave_state_size = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->wave_state, state_bytes));
        ctx->wave_state_size = state_bytes;
    }
    sg::WaveProgress &pr = ctx->wave_progress;
    if (!pr.host) {
        SG_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void **>(&pr.host), sg::kProgressSlots * sizeof(uint2),
                                   cudaHostAllocMapped));
        SG_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void **>(&pr.device), pr.host, 0));
    }
    for (cudaEvent_t &e : pr.done)
        if (!e) SG_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    float4 *base = ctx->wave_state;
    w.state[0] = base;
    w.state[1] = base + (size_t)sg::kWavePlanes * pool;
    w.hits = base + (size_t)2 * sg::kWavePlanes * pool;
    w.ring_queue = reinterpret_cast<uint32_t *>(w.hits + (size_t)sg::kWaveHitPlanes * pool);
    w.surface_queue = w.ring_queue + pool;
    w.counters = reinterpret_cast<sg::WaveCounters *>(w.surface_queue + pool);
    w.progress = pr.device;
    w.pool = pool;
    w.tiles_x = w.tiles_y = 0;
    w.chunk_first = 0;
    return SG_OK;
}

// Sizes the wavefront buffers for a dispatch of `samples` samples and
// fills `w`; the state buffer grows only, the result buffer likewise.
static int ensure_wave(sg_context *ctx, uint32_t samples, sg::WaveParams &w) {
    const uint32_t pool = wave_pool_for(ctx, samples, kDefaultWavePool);
    int status = ensure_wave_state(ctx, pool, w);
    if (status != SG_OK) return status;
    ctx->wave_pool = pool;
    const uint32_t pixels = ctx->width * ctx->height;
    const size_t per_sample = (size_t)pixels * sizeof(float4);
    const uint32_t chunk = (uint32_t)std::max<size_t>(1, std::min<size_t>(samples, kWaveResultBudget / per_sample - 1));
    const size_t result_bytes = sg::wave_result_bytes(pixels, chunk);
    if (result_bytes > ctx->wave_results_size) {
        cudaFree(ctx->wave_results);
        ctx->wave_results = nullptr;
        ctx->wave_results_size = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->wave_results, result_bytes));
        ctx->wave_results_size = result_bytes;
    }
    w.results = ctx->wave_results;
    w.totals = ctx->wave_results + (size_t)chunk * pixels;
    w.chunk_samples = chunk;
    w.sky_results = w.sky_totals = nullptr;
    if (sky_on(ctx)) {
        if (result_bytes > ctx->sky_samples_size) {
            cudaFree(ctx->sky_samples);
            ctx->sky_samples = nullptr;
            ctx->sky_samples_size = 0;
            SG_CUDA(ctx, cudaMalloc(&ctx->sky_samples, result_bytes));
            ctx->sky_samples_size = result_bytes;
        }
        w.sky_results = ctx->sky_samples;
        w.sky_totals = ctx->sky_samples + (size_t)chunk * pixels;
    }
    return SG_OK;
}

// Buffers of the staged adjoint for batches of up to `samples` samples.
static int ensure_adjoint(sg_context *ctx, uint32_t samples, sg::WaveParams &w, sg::AdjointWave &x) {
    const uint32_t pool = wave_pool_for(ctx, samples, kDefaultAdjointPool);
    int status = ensure_wave_state(ctx, pool, w);
    if (status != SG_OK) return status;
    const size_t bytes = sg::adjoint_slot_bytes(pool);
    if (bytes > ctx->adjoint_slots_size) {
        cudaFree(ctx->adjoint_slots);
        ctx->adjoint_slots = nullptr;
        ctx->adjoint_slots_size = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->adjoint_slots, bytes));
        ctx->adjoint_slots_size = bytes;
    }
    char *base = static_cast<char *>(ctx->adjoint_slots);
    x.side = reinterpret_cast<float4 *>(base);
    x.queued = reinterpret_cast<uint4 *>(base + (size_t)pool * sg::kAdjointSideVec4 * sizeof(float4));
    x.lists = base + (size_t)pool * (sg::kAdjointSideVec4 * sizeof(float4) + 2u * sizeof(uint4));
    x.free_ring = reinterpret_cast<uint32_t *>(base + sg::adjoint_slot_bytes(pool) - (size_t)pool * sizeof(uint32_t) -
                                               4 * sizeof(uint32_t));
    x.free_ends = x.free_ring + pool;
    return SG_OK;
}

// Automatic exposure (src/pathtracer.rs:883-905, :980-1000): publish the
// controls — the whole state when metering was off, else everything but the
// eased value — then meter the accumulation, on every encode, whether or
// not it added samples. Nothing runs while automatic exposure is off.
static int meter_exposure(sg_context *ctx, cudaStream_t stream) {
    if (!ctx->options.auto_exposure) {
        ctx->exposure_was_enabled = false;
        return SG_OK;
    }
    if (ctx->width == 0 || ctx->height == 0) return SG_OK;
    DeviceGuard guard(ctx->device);
    if (!ctx->exposure) SG_CUDA(ctx, cudaMalloc(&ctx->exposure, sizeof(sg::ExposureState)));
    if (!ctx->histogram) SG_CUDA(ctx, cudaMalloc(&ctx->histogram, sg::kExposureBins * sizeof(uint32_t)));
    // Pageable source: the bytes are staged before the call returns.
    const sg::ExposureState state{ctx->options.exposure, ctx->options.auto_key, ctx->options.auto_percentile, 1.0f,
                                  ctx->options.ev_bias};
    if (ctx->exposure_was_enabled) {
        SG_CUDA(ctx, cudaMemcpyAsync(reinterpret_cast<char *>(ctx->exposure) + sizeof(float), &state.key,
                                     sizeof(state) - sizeof(float), cudaMemcpyHostToDevice, stream));
    } else {
        SG_CUDA(ctx, cudaMemcpyAsync(ctx->exposure, &state, sizeof(state), cudaMemcpyHostToDevice, stream));
    }
    ctx->exposure_was_enabled = true;
    cudaError_t e = sg::launch_exposure(ctx->mean, ctx->width, ctx->height, ctx->histogram, ctx->exposure, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "exposure metering");
    return SG_OK;
}

// The checkpoint buffers of an accumulation: totals for ck_samples samples
// of every pixel and the record budget (by default half the device memory
// left after the totals). A fresh accumulation clears the record count.
static int ensure_checkpoints(sg_context *ctx, cudaStream_t stream) {
    const size_t pixels = (size_t)ctx->width * ctx->height;
    const size_t totals = pixels * ctx->ck_samples * sizeof(float4);
    if (ctx->ck_totals_size < totals) {
        cudaStreamSynchronize(stream);
        cudaFree(ctx->ck_totals);
        ctx->ck_totals = nullptr;
        ctx->ck_totals_size = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->ck_totals, totals));
        ctx->ck_totals_size = totals;
    }
    if (!ctx->ck_count) SG_CUDA(ctx, cudaMalloc(&ctx->ck_count, sizeof(uint32_t)));
    // Records only where a scatter can bring a path to a checkpoint depth;
    // `every` beyond the bounce limit stores the radiance alone.
    if (!ctx->ck_records && checkpoint_records(ctx)) {
        const size_t record = sg::kCheckpointVec4 * sizeof(float4);
        size_t budget = ctx->ck_record_bytes;
        if (budget == 0) {
            size_t free_bytes = 0, total_bytes = 0;
            SG_CUDA(ctx, cudaMemGetInfo(&free_bytes, &total_bytes));
            budget = free_bytes / 2;
        }
        const size_t capacity = std::min<size_t>(budget / record, 0xffffffffu);
        if (capacity == 0) return fail(ctx, SG_ERR_OOM, "no device memory left for vertex checkpoints");
        SG_CUDA(ctx, cudaMalloc(&ctx->ck_records, capacity * record));
        ctx->ck_capacity = (uint32_t)capacity;
    }
    if (ctx->history.samples == 0u) SG_CUDA(ctx, cudaMemsetAsync(ctx->ck_count, 0, sizeof(uint32_t), stream));
    return SG_OK;
}

// Camera rays of frames with at most 32 bodies test only the bodies and
// rings their 16x16 tile can see: the tile masks, into p.camera_cull.
static int camera_cull(sg_context *ctx, const sg_frame *frame, sg::TraceParams &p, cudaStream_t stream) {
    if (frame->n_bodies > 32u || frame->n_bodies == 0u) return SG_OK;
    const size_t tiles = (size_t)((ctx->width + 15u) / 16u) * ((ctx->height + 15u) / 16u);
    if (ctx->camera_cull_tiles < tiles) {
        cudaStreamSynchronize(stream);
        cudaFree(ctx->camera_cull);
        ctx->camera_cull = nullptr;
        ctx->camera_cull_tiles = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->camera_cull, tiles * sizeof(uint2)));
        ctx->camera_cull_tiles = tiles;
    }
    cudaError_t e = sg::launch_camera_cull(p, ctx->camera_cull, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "camera cull masks");
    ctx->launches += 1;
    p.camera_cull = ctx->camera_cull;
    return SG_OK;
}

static int encode_impl(sg_context *ctx, const sg_frame *frame, void *stream_ptr, uint64_t *events) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    int status = validate_frame(ctx, frame);
    if (status != SG_OK) return status;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    update_history(ctx, frame);
    // Avoid counter wrap and loss of integer resolution in f32 weights
    // (src/pathtracer.rs:802-811).
    const uint32_t remaining =
        ctx->options.sample_limit > ctx->history.samples ? ctx->options.sample_limit - ctx->history.samples : 0u;
    const uint32_t count = std::min({ctx->options.samples_per_frame, (uint32_t)SG_MAX_BATCH_SAMPLES, remaining});
    if (events) std::memset(events, 0, SG_EVENT_COUNT * sizeof(uint64_t));
    if (count > 0 && ctx->width > 0 && ctx->height > 0) {
        DeviceGuard guard(ctx->device);
        const sg_settings s = pack_settings(ctx, frame, count);
        status = upload_bodies(ctx, frame, stream);
        if (status != SG_OK) return status;
        sg::TraceParams p = make_params(ctx, s);
        for (uint32_t k = 0; k < frame->n_bodies; ++k)
            if (frame->bodies[k].axis_x[3] >= 0.5f) p.styled = 1u;
        // A backdrop left by an earlier sky (the history has reset since).
        if (!p.sky_on && ctx->backdrop_written) {
            SG_CUDA(ctx, cudaMemsetAsync(ctx->backdrop, 0, (size_t)ctx->width * ctx->height * sizeof(float4), stream));
            ctx->backdrop_written = false;
        }
        if (p.sky_on) ctx->backdrop_written = true;
        // The surface sky cache, built by an accumulation's first dispatch
        // (src/pathtracer.rs:946-954).
        if (p.air_on) {
            if (!ctx->sky_light) {
                SG_CUDA(ctx, cudaMalloc(&ctx->sky_light, sg::kSkyCacheTexels * sizeof(float4)));
                p.sky_light = ctx->sky_light;
            }
            if (ctx->history.samples == 0u) {
                cudaError_t e = sg::launch_sky_cache(p, ctx->sky_light, stream);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "surface sky cache");
                ctx->launches += 1;
            }
        }
        if (events) {
            SG_CUDA(ctx, cudaMemsetAsync(ctx->events, 0, sg::kEventCount * sizeof(unsigned long long), stream));
            p.events = ctx->events;
        } else {
            status = camera_cull(ctx, frame, p, stream);
            if (status != SG_OK) return status;
        }
        const bool checkpointing = ctx->ck_every > 0u && !events && ctx->integrator == SG_INTEGRATOR_WAVEFRONT &&
                                   !p.air_on && !p.styled && !p.sky_on;
        if (ctx->history.samples == 0u) ctx->ck_valid = checkpointing;
        if (!checkpointing) ctx->ck_valid = false;
        if (!events && ctx->integrator == SG_INTEGRATOR_WAVEFRONT) {
            sg::WaveParams w{};
            status = ensure_wave(ctx, count, w);
            if (status != SG_OK) return status;
            if (ctx->ck_valid) {
                status = ensure_checkpoints(ctx, stream);
                if (status != SG_OK) return status;
                w.ck.records = checkpoint_records(ctx) ? ctx->ck_records : nullptr;
                w.ck.count = ctx->ck_count;
                w.ck.capacity = ctx->ck_capacity;
                w.ck.totals = ctx->ck_totals;
                w.ck.samples = ctx->ck_samples;
                w.ck.sample_base = ctx->history.samples;
                w.ck.every = ctx->ck_every;
                w.ck.max_depth = ctx->options.max_bounces;
            }
            sg::WaveRun run;
            sg::StageMarks *marks = ctx->stage_timing ? &ctx->stage_marks : nullptr;
            cudaError_t e = sg::launch_wavefront(p, w, ctx->wave_progress, stream, &run, marks);
            ctx->wave_iterations = run.iterations;
            ctx->launches += run.kernels;
            if (e == cudaErrorLaunchTimeout)
                return fail(ctx, SG_ERR_TIMEOUT, "wavefront dispatch did not drain within its iteration bound");
            if (e != cudaSuccess) return cuda_fail(ctx, e, "wavefront dispatch");
            if (marks && marks->used > 0) {
                SG_CUDA(ctx, cudaEventSynchronize(marks->events[marks->used - 1]));
                for (float &v : ctx->stage_ms) v = 0.0f;
                for (size_t k = 0; k + 1 < marks->used; ++k) {
                    float ms = 0.0f;
                    SG_CUDA(ctx, cudaEventElapsedTime(&ms, marks->events[k], marks->events[k + 1]));
                    ctx->stage_ms[marks->stage[k]] += ms;
                }
            }
        } else {
            cudaError_t e = sg::launch_trace(p, events != nullptr, stream);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
            ctx->launches += 1;
        }
        record_run(ctx, s.sampling[0], count);
        if (events) {
            unsigned long long host[sg::kEventCount];
            SG_CUDA(ctx, cudaMemcpyAsync(host, ctx->events, sizeof(host), cudaMemcpyDeviceToHost, stream));
            SG_CUDA(ctx, cudaStreamSynchronize(stream));
            for (int k = 0; k < sg::kEventCount; ++k) events[k] = host[k];
        }
    }
    status = meter_exposure(ctx, stream);
    if (status != SG_OK) return status;
    ctx->history.samples += count;
    ctx->history.sequence += count;
    ctx->exposure_idle_frames = count > 0 ? 0u : (ctx->exposure_idle_frames == UINT32_MAX ? UINT32_MAX : ctx->exposure_idle_frames + 1u);
    return SG_OK;
}

int sg_encode(sg_context *ctx, const sg_frame *frame, void *stream_ptr) {
    return encode_impl(ctx, frame, stream_ptr, nullptr);
}

int sg_encode_counted(sg_context *ctx, const sg_frame *frame, void *stream_ptr, uint64_t *events) {
    if (!events) return fail(ctx, SG_ERR_INVALID, "events is NULL");
    return encode_impl(ctx, frame, stream_ptr, events);
}

int sg_measure_fp32_peak(int device, double *flops_per_second) {
    if (!flops_per_second) return fail(nullptr, SG_ERR_INVALID, "flops_per_second is NULL");
    DeviceGuard guard(device);
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaDeviceGetAttribute");
    float *out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(float))) != cudaSuccess) return cuda_fail(nullptr, e, "cudaMalloc");
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, iters = 4096;
    double best = 0.0;
    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
        cudaEventRecord(a, nullptr);
        e = sg::launch_fma_peak(blocks, iters, out, nullptr);
        cudaEventRecord(b, nullptr);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float ms = 0.0f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, a, b);
        const double flops = 2.0 * 128.0 * iters * 256.0 * blocks;
        if (rep > 0 && ms > 0.0f) best = std::max(best, flops / (ms * 1e-3));
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(out);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "fma peak kernel");
    *flops_per_second = best;
    return SG_OK;
}

int sg_get_samples(const sg_context *ctx, uint32_t *samples, uint32_t *sequence) {
    if (!ctx) return SG_ERR_INVALID;
    if (samples) *samples = ctx->history.samples;
    if (sequence) *sequence = ctx->history.sequence;
    return SG_OK;
}

int sg_needs_redraw(const sg_context *ctx, int *redraw) {
    if (!ctx || !redraw) return SG_ERR_INVALID;
    *redraw = ctx->history.samples < ctx->options.sample_limit ||
              (ctx->options.auto_exposure && ctx->exposure_idle_frames < 60u);
    return SG_OK;
}

int sg_get_size(const sg_context *ctx, uint32_t *width, uint32_t *height) {
    if (!ctx) return SG_ERR_INVALID;
    if (width) *width = ctx->width;
    if (height) *height = ctx->height;
    return SG_OK;
}

static int read_image(sg_context *ctx, const float4 *src, float *dst, int on_device, void *stream_ptr) {
    if (!ctx || !dst) return fail(ctx, SG_ERR_INVALID, "ctx or dst is NULL");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t bytes = (size_t)ctx->width * ctx->height * sizeof(float4);
    if (bytes == 0) return SG_OK;
    SG_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                                 stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    return SG_OK;
}

int sg_read_accumulation(sg_context *ctx, float *dst, int dst_on_device, void *stream) {
    return read_image(ctx, ctx ? ctx->mean : nullptr, dst, dst_on_device, stream);
}

int sg_read_backdrop(sg_context *ctx, float *dst, int dst_on_device, void *stream) {
    return read_image(ctx, ctx ? ctx->backdrop : nullptr, dst, dst_on_device, stream);
}

int sg_set_accumulation(sg_context *ctx, const float *src, int src_on_device, uint32_t samples,
                        uint32_t sequence, void *stream_ptr) {
    if (!ctx || !src) return fail(ctx, SG_ERR_INVALID, "ctx or src is NULL");
    if (samples > SG_MAX_SAMPLES) return fail(ctx, SG_ERR_INVALID, "samples exceed the f32 weight limit");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t n = (size_t)ctx->width * ctx->height;
    if (n == 0) return SG_OK;
    std::vector<float> host(n * 4);
    if (src_on_device) {
        SG_CUDA(ctx, cudaMemcpyAsync(host.data(), src, n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
        SG_CUDA(ctx, cudaStreamSynchronize(stream));
    } else {
        std::memcpy(host.data(), src, n * sizeof(float4));
    }
    // The compensated sum restarts from mean * samples.
    std::vector<float> sums(n * 4);
    for (size_t k = 0; k < n * 4; ++k) sums[k] = host[k] * (float)samples;
    SG_CUDA(ctx, cudaMemcpyAsync(ctx->mean, host.data(), n * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SG_CUDA(ctx, cudaMemcpyAsync(ctx->sum, sums.data(), n * sizeof(float4), cudaMemcpyHostToDevice, stream));
    SG_CUDA(ctx, cudaMemsetAsync(ctx->comp, 0, n * sizeof(float4), stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    ctx->history.samples = samples;
    ctx->history.sequence = sequence;
    // The restored samples' noise keys are unknown: no replay.
    ctx->history.runs.clear();
    ctx->history.replayable = samples == 0;
    return SG_OK;
}

int sg_accumulation_device_ptr(sg_context *ctx, void **ptr) {
    if (!ctx || !ptr) return SG_ERR_INVALID;
    *ptr = ctx->mean;
    return SG_OK;
}

int sg_upload_ring_profile(sg_context *ctx, uint32_t slot, const float *tau, uint32_t bins) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (slot >= SG_RING_TABLE_SLOTS) return fail(ctx, SG_ERR_INVALID, "ring-table slot out of range");
    if (bins > SG_RING_TABLE_MAX_BINS) return fail(ctx, SG_ERR_CAPACITY, "too many ring-table bins");
    if (bins > 0 && !tau) return fail(ctx, SG_ERR_INVALID, "tau is NULL");
    for (uint32_t k = 0; k < bins; ++k)
        if (!(tau[k] >= 0.0f) || !std::isfinite(tau[k]))
            return fail(ctx, SG_ERR_INVALID, "ring optical depths must be finite and non-negative");
    DeviceGuard guard(ctx->device);
    if (bins)
        SG_CUDA(ctx, cudaMemcpy(ctx->ring_tables + (size_t)slot * SG_RING_TABLE_MAX_BINS, tau, bins * sizeof(float),
                                cudaMemcpyHostToDevice));
    ctx->ring_bins[slot] = bins;
    ctx->table_version += 1;
    return SG_OK;
}

// Shared set-up of the probe entry points: settings as encode would pack
// them (without touching the history), bodies uploaded.
static int probe_setup(sg_context *ctx, const sg_frame *frame, cudaStream_t stream, sg::TraceParams *p) {
    int status = validate_frame(ctx, frame);
    if (status != SG_OK) return status;
    const sg_settings s = pack_settings(ctx, frame, 0);
    status = upload_bodies(ctx, frame, stream);
    if (status != SG_OK) return status;
    *p = make_params(ctx, s);
    return SG_OK;
}

int sg_closest_hit(sg_context *ctx, const sg_frame *frame, const sg_ray *rays, uint32_t n, sg_hit *hits,
                   int on_device, void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (n && (!rays || !hits)) return fail(ctx, SG_ERR_INVALID, "rays or hits is NULL");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    sg::TraceParams p;
    int status = probe_setup(ctx, frame, stream, &p);
    if (status != SG_OK || n == 0) return status;
    const sg_ray *d_rays = rays;
    sg_hit *d_hits = hits;
    if (!on_device) {
        status = ensure_scratch(ctx, (size_t)n * (sizeof(sg_ray) + sizeof(sg_hit)) + 256);
        if (status != SG_OK) return status;
        d_rays = static_cast<const sg_ray *>(ctx->scratch);
        d_hits = reinterpret_cast<sg_hit *>(static_cast<char *>(ctx->scratch) + (((size_t)n * sizeof(sg_ray) + 255) & ~size_t(255)));
        SG_CUDA(ctx, cudaMemcpyAsync((void *)d_rays, rays, n * sizeof(sg_ray), cudaMemcpyHostToDevice, stream));
    }
    cudaError_t e = sg::launch_closest_hit(p, d_rays, d_hits, n, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "closest_hit launch");
    if (!on_device) SG_CUDA(ctx, cudaMemcpyAsync(hits, d_hits, n * sizeof(sg_hit), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    return SG_OK;
}

int sg_light_visibility(sg_context *ctx, const sg_frame *frame, const sg_ray *rays, const uint32_t *lights,
                        uint32_t n, float *out, int on_device, void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (n && (!rays || !lights || !out)) return fail(ctx, SG_ERR_INVALID, "rays, lights or out is NULL");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    sg::TraceParams p;
    int status = probe_setup(ctx, frame, stream, &p);
    if (status != SG_OK || n == 0) return status;
    const sg_ray *d_rays = rays;
    const uint32_t *d_lights = lights;
    float *d_out = out;
    if (!on_device) {
        const size_t ray_bytes = ((size_t)n * sizeof(sg_ray) + 255) & ~size_t(255);
        const size_t light_bytes = ((size_t)n * sizeof(uint32_t) + 255) & ~size_t(255);
        status = ensure_scratch(ctx, ray_bytes + light_bytes + (size_t)n * sizeof(float));
        if (status != SG_OK) return status;
        char *base = static_cast<char *>(ctx->scratch);
        d_rays = reinterpret_cast<const sg_ray *>(base);
        d_lights = reinterpret_cast<const uint32_t *>(base + ray_bytes);
        d_out = reinterpret_cast<float *>(base + ray_bytes + light_bytes);
        SG_CUDA(ctx, cudaMemcpyAsync((void *)d_rays, rays, n * sizeof(sg_ray), cudaMemcpyHostToDevice, stream));
        SG_CUDA(ctx, cudaMemcpyAsync((void *)d_lights, lights, n * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    }
    cudaError_t e = sg::launch_light_visibility(p, d_rays, d_lights, d_out, n, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "light_visibility launch");
    if (!on_device) SG_CUDA(ctx, cudaMemcpyAsync(out, d_out, n * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    return SG_OK;
}

int sg_ring_probe(sg_context *ctx, const sg_frame *frame, const sg_ray *rays, uint32_t body, uint32_t n, float *out,
                  int on_device, void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (n && (!rays || !out)) return fail(ctx, SG_ERR_INVALID, "rays or out is NULL");
    if (frame && body >= frame->n_bodies) return fail(ctx, SG_ERR_INVALID, "body index out of range");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    sg::TraceParams p;
    int status = probe_setup(ctx, frame, stream, &p);
    if (status != SG_OK || n == 0) return status;
    const sg_ray *d_rays = rays;
    float *d_out = out;
    if (!on_device) {
        const size_t ray_bytes = ((size_t)n * sizeof(sg_ray) + 255) & ~size_t(255);
        status = ensure_scratch(ctx, ray_bytes + (size_t)n * sizeof(float4));
        if (status != SG_OK) return status;
        char *base = static_cast<char *>(ctx->scratch);
        d_rays = reinterpret_cast<const sg_ray *>(base);
        d_out = reinterpret_cast<float *>(base + ray_bytes);
        SG_CUDA(ctx, cudaMemcpyAsync((void *)d_rays, rays, n * sizeof(sg_ray), cudaMemcpyHostToDevice, stream));
    }
    cudaError_t e = sg::launch_ring_probe(p, d_rays, body, d_out, n, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ring_probe launch");
    if (!on_device) SG_CUDA(ctx, cudaMemcpyAsync(out, d_out, n * sizeof(float4), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    return SG_OK;
}

int sg_terrain_probe(sg_context *ctx, const sg_frame *frame, const float *rays, uint32_t n, float *out, int on_device,
                     void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (n && (!rays || !out)) return fail(ctx, SG_ERR_INVALID, "rays or out is NULL");
    if (!ctx->terrain) return fail(ctx, SG_ERR_STATE, "no terrain was uploaded");
    if (frame && frame->globals && (frame->globals->ground_north[3] == 0.0f || frame->globals->ground_counts[1] == 0u))
        return fail(ctx, SG_ERR_INVALID, "the frame must enable the landscape and its terrain");
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    sg::TraceParams p;
    int status = probe_setup(ctx, frame, stream, &p);
    if (status != SG_OK || n == 0) return status;
    const float *d_rays = rays;
    float *d_out = out;
    if (!on_device) {
        const size_t ray_bytes = ((size_t)n * 6 * sizeof(float) + 255) & ~size_t(255);
        status = ensure_scratch(ctx, ray_bytes + (size_t)n * 4 * sizeof(float));
        if (status != SG_OK) return status;
        char *base = static_cast<char *>(ctx->scratch);
        d_rays = reinterpret_cast<const float *>(base);
        d_out = reinterpret_cast<float *>(base + ray_bytes);
        SG_CUDA(ctx, cudaMemcpyAsync((void *)d_rays, rays, (size_t)n * 6 * sizeof(float), cudaMemcpyHostToDevice, stream));
    }
    cudaError_t e = sg::launch_terrain_probe(p, d_rays, d_out, n, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "terrain_probe launch");
    if (!on_device)
        SG_CUDA(ctx, cudaMemcpyAsync(out, d_out, (size_t)n * 4 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    return SG_OK;
}

int sg_ring_energy(sg_context *ctx, float albedo, float tau, float mu, uint32_t steps, float *energy) {
    if (!ctx || !energy) return fail(ctx, SG_ERR_INVALID, "ctx or energy is NULL");
    if (!(mu > 0.0f) || steps == 0 || steps > (1u << 20))
        return fail(ctx, SG_ERR_INVALID, "mu must be positive and steps in 1..2^20");
    DeviceGuard guard(ctx->device);
    int status = ensure_scratch(ctx, sizeof(float));
    if (status != SG_OK) return status;
    float *d = static_cast<float *>(ctx->scratch);
    cudaError_t e = sg::launch_ring_energy(albedo, tau, mu, steps, d, nullptr);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "ring_energy launch");
    SG_CUDA(ctx, cudaMemcpy(energy, d, sizeof(float), cudaMemcpyDeviceToHost));
    return SG_OK;
}

int sg_set_integrator(sg_context *ctx, int integrator, uint32_t pool_paths) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (integrator != SG_INTEGRATOR_MEGAKERNEL && integrator != SG_INTEGRATOR_WAVEFRONT)
        return fail(ctx, SG_ERR_INVALID, "unknown integrator");
    if (pool_paths != 0 && (pool_paths < 256u || pool_paths > SG_WAVE_MAX_POOL))
        return fail(ctx, SG_ERR_INVALID, "pool_paths must be 0 or in 256..SG_WAVE_MAX_POOL");
    ctx->integrator = integrator;
    ctx->wave_pool_request = pool_paths;
    return SG_OK;
}

int sg_get_integrator(const sg_context *ctx, int *integrator, uint32_t *pool_paths, uint32_t *iterations) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (integrator) *integrator = ctx->integrator;
    if (pool_paths) *pool_paths = ctx->wave_pool;
    if (iterations) *iterations = ctx->wave_iterations;
    return SG_OK;
}

static_assert(sg::kStageCount == SG_STAGE_COUNT, "stage count");

int sg_display(sg_context *ctx, uint32_t width, uint32_t height, int format, void *out, int on_device,
               void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (!out) return fail(ctx, SG_ERR_INVALID, "out is NULL");
    if (format != SG_DISPLAY_RGBA8_SRGB && format != SG_DISPLAY_RGBA32F)
        return fail(ctx, SG_ERR_INVALID, "format must be SG_DISPLAY_RGBA8_SRGB or SG_DISPLAY_RGBA32F");
    if (width == 0 || height == 0 || width > 16384 || height > 16384)
        return fail(ctx, SG_ERR_INVALID, "display size must be 1..16384 on each side");
    if (ctx->width == 0 || ctx->height == 0) return fail(ctx, SG_ERR_STATE, "the context has no viewport");
    const bool automatic = ctx->options.auto_exposure && ctx->exposure_was_enabled;
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t bytes = (size_t)width * height * (format == SG_DISPLAY_RGBA32F ? 16u : 4u);
    void *dst = out;
    if (!on_device) {
        int status = ensure_scratch(ctx, bytes);
        if (status != SG_OK) return status;
        dst = ctx->scratch;
    }
    sg::DisplayParams d{};
    d.mean = ctx->mean;
    d.backdrop = ctx->backdrop;
    d.width = ctx->width;
    d.height = ctx->height;
    d.out_width = width;
    d.out_height = height;
    d.format = format;
    d.out = dst;
    d.automatic = automatic ? 1 : 0;
    d.state = ctx->exposure;
    d.manual = ctx->options.exposure;
    d.bias = ctx->options.ev_bias;
    d.milky_way = ctx->options.milky_way;
    cudaError_t e = sg::launch_display(d, stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "display");
    if (!on_device) {
        SG_CUDA(ctx, cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, stream));
        SG_CUDA(ctx, cudaStreamSynchronize(stream));
    }
    return SG_OK;
}

int sg_set_exposure_controls(sg_context *ctx, int automatic, float bias) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (!std::isfinite(bias)) return fail(ctx, SG_ERR_INVALID, "bias must be finite");
    ctx->options.auto_exposure = automatic ? 1 : 0;
    ctx->options.ev_bias = bias;
    ctx->exposure_idle_frames = 0;
    return SG_OK;
}

int sg_get_exposure(sg_context *ctx, float *exposure, void *stream_ptr) {
    if (!ctx || !exposure) return fail(ctx, SG_ERR_INVALID, "ctx or exposure is NULL");
    if (!(ctx->options.auto_exposure && ctx->exposure_was_enabled && ctx->exposure)) {
        *exposure = ctx->options.exposure;
        return SG_OK;
    }
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    float value = 0.0f;
    SG_CUDA(ctx, cudaMemcpyAsync(&value, ctx->exposure, sizeof(float), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    *exposure = value;
    return SG_OK;
}

int sg_set_stage_timing(sg_context *ctx, int enable) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    ctx->stage_timing = enable != 0;
    return SG_OK;
}

int sg_get_stage_times(const sg_context *ctx, float *ms) {
    if (!ctx || !ms) return fail(nullptr, SG_ERR_INVALID, "ctx or ms is NULL");
    for (int k = 0; k < sg::kStageCount; ++k) ms[k] = ctx->stage_ms[k];
    return SG_OK;
}

int sg_set_fp64_sites(sg_context *ctx, int enable) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    ctx->fp64_sites = enable != 0;
    return SG_OK;
}

int sg_set_guided_ground(sg_context *ctx, int enable) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    ctx->guided_ground = enable != 0;
    return SG_OK;
}

int sg_set_checkpoints(sg_context *ctx, uint32_t every, uint32_t max_samples, uint64_t record_bytes) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (every > 64u) return fail(ctx, SG_ERR_INVALID, "every must be in 0..64");
    if (every > 0u && (max_samples == 0u || max_samples > SG_MAX_SAMPLES))
        return fail(ctx, SG_ERR_INVALID, "max_samples must be in 1..SG_MAX_SAMPLES");
    DeviceGuard guard(ctx->device);
    cudaDeviceSynchronize();
    cudaFree(ctx->ck_records);
    cudaFree(ctx->ck_totals);
    ctx->ck_records = nullptr;
    ctx->ck_totals = nullptr;
    ctx->ck_totals_size = 0;
    ctx->ck_capacity = 0;
    ctx->ck_every = every;
    ctx->ck_samples = every > 0u ? max_samples : 0u;
    ctx->ck_record_bytes = record_bytes;
    ctx->ck_valid = false;
    return SG_OK;
}

int sg_get_checkpoint_stats(sg_context *ctx, uint64_t *device_bytes, uint64_t *records, uint64_t *dropped) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    uint32_t claimed = 0;
    if (ctx->ck_count) {
        DeviceGuard guard(ctx->device);
        SG_CUDA(ctx, cudaMemcpy(&claimed, ctx->ck_count, sizeof(claimed), cudaMemcpyDeviceToHost));
    }
    const uint64_t stored = std::min<uint64_t>(claimed, ctx->ck_capacity);
    if (device_bytes)
        *device_bytes = ctx->ck_totals_size + stored * sg::kCheckpointVec4 * sizeof(float4) + (ctx->ck_count ? 4u : 0u);
    if (records) *records = stored;
    if (dropped) *dropped = claimed - stored;
    return SG_OK;
}

int sg_set_ringshine(sg_context *ctx, int enable) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    ctx->ringshine = enable != 0;
    return SG_OK;
}

int sg_get_tape(const sg_context *ctx, sg_tape *tape) {
    if (!ctx || !tape) return fail(nullptr, SG_ERR_INVALID, "ctx or tape is NULL");
    if (!ctx->history.replayable)
        return fail(const_cast<sg_context *>(ctx), SG_ERR_STATE,
                    "the accumulation was restored or mixes too many noise runs and cannot be replayed");
    std::memset(tape, 0, sizeof(*tape));
    tape->width = ctx->width;
    tape->height = ctx->height;
    tape->samples = ctx->history.samples;
    tape->n_ranges = (uint32_t)ctx->history.runs.size();
    for (size_t k = 0; k < ctx->history.runs.size(); ++k) {
        tape->first[k] = ctx->history.runs[k].first;
        tape->count[k] = ctx->history.runs[k].second;
    }
    tape->history_hash = ctx->history.key_hash;
    return SG_OK;
}

int sg_backward(sg_context *ctx, const sg_frame *frame, const sg_tape *tape, const float *dl_dimage, int on_device,
                sg_gradients *grads, void *stream_ptr) {
    if (!ctx) return fail(nullptr, SG_ERR_INVALID, "ctx is NULL");
    if (!tape || !dl_dimage || !grads) return fail(ctx, SG_ERR_INVALID, "tape, dl_dimage or grads is NULL");
    if (tape->width != ctx->width || tape->height != ctx->height)
        return fail(ctx, SG_ERR_STATE, "the tape was recorded at another viewport size");
    if (tape->n_ranges > SG_TAPE_RANGES) return fail(ctx, SG_ERR_INVALID, "tape n_ranges exceeds SG_TAPE_RANGES");
    uint64_t total = 0;
    for (uint32_t k = 0; k < tape->n_ranges; ++k) total += tape->count[k];
    if (total != tape->samples || total == 0 || total > SG_MAX_SAMPLES)
        return fail(ctx, SG_ERR_INVALID, "tape runs must hold 1..SG_MAX_SAMPLES samples in total");
    int status = validate_frame(ctx, frame);
    if (status != SG_OK) return status;
    if (sky_on(ctx))
        return fail(ctx, SG_ERR_STATE, "the adjoint does not differentiate the sky backdrop; remove the catalogue and panorama");
    if (frame->globals->atmo_params[3] >= 0.5f)
        return fail(ctx, SG_ERR_STATE, "the adjoint does not differentiate the host air (atmo_params.w >= 0.5)");
    for (uint32_t i = 0; i < frame->n_bodies; ++i)
        if (frame->bodies[i].axis_x[3] >= 0.5f)
            return fail(ctx, SG_ERR_STATE, "the adjoint does not differentiate procedural surface styles (axis_x.w >= 0.5)");
    if (key_hash(history_key(ctx, frame)) != tape->history_hash)
        return fail(ctx, SG_ERR_STATE, "frame, options or tables differ from the ones the tape was recorded with");
    grads->dropped = 0;
    const size_t pixels = (size_t)ctx->width * ctx->height;
    if (pixels == 0) return SG_OK;
    DeviceGuard guard(ctx->device);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    const size_t texels = ctx->albedo_map ? (size_t)ctx->map_width * ctx->map_height : 0;
    const size_t floats = sg::kGradMap + texels;
    if (ctx->grad_floats < floats) {
        cudaStreamSynchronize(stream);
        cudaFree(ctx->grad);
        ctx->grad = nullptr;
        ctx->grad_floats = 0;
        SG_CUDA(ctx, cudaMalloc(&ctx->grad, floats * sizeof(float)));
        ctx->grad_floats = floats;
    }
    if (!ctx->dropped) SG_CUDA(ctx, cudaMalloc(&ctx->dropped, sizeof(unsigned long long)));
    const float4 *d_dl = reinterpret_cast<const float4 *>(dl_dimage);
    if (!on_device) {
        if (ctx->dl_pixels < pixels) {
            cudaStreamSynchronize(stream);
            cudaFree(ctx->dl_dimage);
            ctx->dl_dimage = nullptr;
            ctx->dl_pixels = 0;
            SG_CUDA(ctx, cudaMalloc(&ctx->dl_dimage, pixels * sizeof(float4)));
            ctx->dl_pixels = pixels;
        }
        SG_CUDA(ctx, cudaMemcpyAsync(ctx->dl_dimage, dl_dimage, pixels * sizeof(float4), cudaMemcpyHostToDevice, stream));
        d_dl = ctx->dl_dimage;
    }
    SG_CUDA(ctx, cudaMemsetAsync(ctx->grad, 0, floats * sizeof(float), stream));
    SG_CUDA(ctx, cudaMemsetAsync(ctx->dropped, 0, sizeof(unsigned long long), stream));
    sg_settings s = pack_settings(ctx, frame, 0);
    status = upload_bodies(ctx, frame, stream);
    if (status != SG_OK) return status;
    sg::AdjointParams a;
    a.dl_dimage = d_dl;
    a.inv_samples = 1.0f / (float)tape->samples;
    a.grad = ctx->grad;
    a.overflow = ctx->dropped;
    // Shared-memory windows: the used ring-table range (when it is small)
    // and the per-body colours.
    uint32_t tau_used = 0;
    for (uint32_t k = 0; k < SG_RING_TABLE_SLOTS; ++k)
        if (ctx->ring_bins[k]) tau_used = k * SG_RING_TABLE_MAX_BINS + ctx->ring_bins[k];
    a.tau_window = tau_used <= 8192u ? tau_used : 0u;
    a.color_window = 6u * frame->n_bodies;
    a.ck = sg::Checkpoints{};
    // With vertex checkpoints of this accumulation, the replay (staged or
    // per-pixel) takes each sample, its radiance known, only up to its first
    // checkpoint, and the segment kernel replays the rest from the records.
    const bool checkpointed = ctx->ck_every > 0u && ctx->ck_valid && ctx->ck_totals;
    uint32_t records = 0;
    if (checkpointed) {
        if (ctx->ck_records) {
            uint32_t claimed = 0;
            SG_CUDA(ctx, cudaMemcpyAsync(&claimed, ctx->ck_count, sizeof(claimed), cudaMemcpyDeviceToHost, stream));
            SG_CUDA(ctx, cudaStreamSynchronize(stream));
            records = std::min(claimed, ctx->ck_capacity);
        }
        a.ck.records = ctx->ck_records;
        a.ck.count = ctx->ck_count;
        a.ck.capacity = ctx->ck_capacity;
        a.ck.totals = ctx->ck_totals;
        a.ck.samples = ctx->ck_samples;
        a.ck.every = ctx->ck_every;
        a.ck.max_depth = ctx->options.max_bounces;
    }
    const bool staged = ctx->integrator == SG_INTEGRATOR_WAVEFRONT;
    sg::WaveParams w{};
    sg::AdjointWave x{};
    if (staged) {
        uint32_t largest = 0;
        for (uint32_t k = 0; k < tape->n_ranges; ++k)
            largest = std::max(largest, std::min<uint32_t>(SG_MAX_BATCH_SAMPLES, tape->count[k]));
        status = ensure_adjoint(ctx, largest, w, x);
        if (status != SG_OK) return status;
        cudaError_t e = sg::reset_adjoint_slots(x, w.pool, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint slot reset");
    }
    uint32_t accumulated = 0;  // accumulation index of the launch's first sample
    for (uint32_t k = 0; k < tape->n_ranges; ++k) {
        for (uint32_t done = 0; done < tape->count[k]; done += SG_MAX_BATCH_SAMPLES) {
            s.sampling[0] = tape->first[k] + done;
            s.counts[2] = std::min<uint32_t>(SG_MAX_BATCH_SAMPLES, tape->count[k] - done);
            a.ck.sample_base = accumulated;
            accumulated += s.counts[2];
            sg::TraceParams p = make_params(ctx, s);
            status = camera_cull(ctx, frame, p, stream);
            if (status != SG_OK) return status;
            if (staged) {
                sg::WaveRun run;
                cudaError_t e = sg::launch_adjoint_wavefront(p, a, w, x, ctx->wave_progress, stream, &run);
                ctx->launches += run.kernels;
                if (e == cudaErrorLaunchTimeout)
                    return fail(ctx, SG_ERR_TIMEOUT, "staged adjoint did not drain within its iteration bound");
                if (e != cudaSuccess) return cuda_fail(ctx, e, "staged adjoint");
            } else {
                cudaError_t e = sg::launch_adjoint(p, a, stream);
                if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint launch");
                ctx->launches += 1;
            }
        }
    }
    if (checkpointed && records > 0) {
        const sg::TraceParams p = make_params(ctx, s);
        cudaError_t e = sg::launch_checkpoint_segments(p, a, records, stream);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "checkpoint segments");
        ctx->launches += 1;
    }
    const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    if (grads->ring_tau)
        SG_CUDA(ctx, cudaMemcpyAsync(grads->ring_tau, ctx->grad, sg::kGradColor * sizeof(float), kind, stream));
    const float *colors = ctx->grad + sg::kGradColor;
    if (grads->ring_albedo && frame->n_bodies)
        SG_CUDA(ctx, cudaMemcpy2DAsync(grads->ring_albedo, 3 * sizeof(float), colors, 6 * sizeof(float),
                                       3 * sizeof(float), frame->n_bodies, kind, stream));
    if (grads->body_color && frame->n_bodies)
        SG_CUDA(ctx, cudaMemcpy2DAsync(grads->body_color, 3 * sizeof(float), colors + 3, 6 * sizeof(float),
                                       3 * sizeof(float), frame->n_bodies, kind, stream));
    if (grads->albedo_map && texels)
        SG_CUDA(ctx, cudaMemcpyAsync(grads->albedo_map, ctx->grad + sg::kGradMap, texels * sizeof(float), kind,
                                     stream));
    unsigned long long dropped = 0;
    SG_CUDA(ctx, cudaMemcpyAsync(&dropped, ctx->dropped, sizeof(dropped), cudaMemcpyDeviceToHost, stream));
    SG_CUDA(ctx, cudaStreamSynchronize(stream));
    grads->dropped = dropped;
    return SG_OK;
}

}  // extern "C"

void sg::set_library_error(const char *message) { g_last_error = message ? message : ""; }

extern "C" {

const char *sg_last_error(const sg_context *ctx) {
    if (ctx) return ctx->last_error.c_str();
    return g_last_error.c_str();
}

const char *sg_status_string(int status) {
    switch (status) {
        case SG_OK: return "ok";
        case SG_ERR_INVALID: return "invalid argument";
        case SG_ERR_CAPACITY: return "capacity exceeded";
        case SG_ERR_CUDA: return "CUDA error";
        case SG_ERR_OOM: return "out of device memory";
        case SG_ERR_STATE: return "invalid state";
        case SG_ERR_TIMEOUT: return "device loop gave up";
        default: return "unknown status";
    }
}

int sg_launch_count(const sg_context *ctx, uint64_t *launches) {
    if (!ctx || !launches) return SG_ERR_INVALID;
    *launches = ctx->launches;
    return SG_OK;
}

}  // extern "C"
