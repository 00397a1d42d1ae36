// sg_noalloc.cu — closest-hit queries that allocate no device memory.
//
// sg_closest_hit stages host rays and hits in a buffer owned by the context,
// which it grows with cudaMalloc when a query is larger than the last one.
// Some callers cannot let the library allocate at query time: a host
// application that hands the whole device to its own allocator (a caching
// allocator or a memory pool sized to all free memory), where a library
// cudaMalloc fails or splits the pool; and latency-bound callers, for which
// cudaMalloc and cudaFree are too slow and synchronise the device. For them
// sg_closest_hit_noalloc stages the frame's bodies, the rays and the hits in
// one fixed file-scope device array instead, and needs no context either.
//
// The array is SG_NOALLOC_SCRATCH_BYTES; every GPU that loads the library
// holds it until the process exits. Every call on a device uses the same
// array, so calls whose work overlaps on the GPU (two host threads, or two
// streams) race. Nothing in it has to start at zero: each call copies in
// its bodies and rays, and the kernel writes every hit before it is read.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/stargaze_b200.h"
#include "sg_internal.h"

namespace {

constexpr size_t align256(size_t bytes) { return (bytes + 255u) & ~size_t(255u); }

// Layout of the array: bodies, then rays, then hits, each 256-byte aligned.
constexpr size_t kBodiesOffset = 0;
constexpr size_t kRaysOffset = align256(kBodiesOffset + SG_BODY_CAPACITY * sizeof(sg_sphere));
constexpr size_t kHitsOffset = align256(kRaysOffset + (size_t)SG_NOALLOC_MAX_RAYS * sizeof(sg_ray));
constexpr size_t kScratchEnd = kHitsOffset + (size_t)SG_NOALLOC_MAX_RAYS * sizeof(sg_hit);
static_assert(kScratchEnd <= SG_NOALLOC_SCRATCH_BYTES, "the staging layout must fit the array");

static __device__ __align__(256) unsigned char scratch[SG_NOALLOC_SCRATCH_BYTES];

// The array's device address, looked up once per device. In host code the
// name `scratch` is only a host-side handle; a kernel must get this address.
constexpr int kMaxDevices = 64;
std::mutex g_lock;
unsigned char *g_address[kMaxDevices] = {};

int fail(int status, const char *message) {
    sg::set_library_error(message);
    return status;
}

int cuda_fail(cudaError_t e, const char *what) {
    char message[256];
    std::snprintf(message, sizeof(message), "%s: %s", what, cudaGetErrorString(e));
    sg::set_library_error(message);
    return e == cudaErrorMemoryAllocation ? SG_ERR_OOM : SG_ERR_CUDA;
}

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

// With `device` current: the array's address on it (set-up on first use).
int scratch_address(int device, unsigned char **out) {
    std::lock_guard<std::mutex> hold(g_lock);
    if (!g_address[device]) {
        void *address = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&address, scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress");
        g_address[device] = static_cast<unsigned char *>(address);
    }
    *out = g_address[device];
    return SG_OK;
}

}  // namespace

extern "C" int sg_closest_hit_noalloc(int device, const sg_frame *frame, const sg_ray *rays, uint32_t n,
                                      sg_hit *hits, void *stream_ptr) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count || device >= kMaxDevices) return fail(SG_ERR_INVALID, "no such CUDA device");
    if (!frame || !frame->globals) return fail(SG_ERR_INVALID, "frame or frame->globals is NULL");
    if (frame->n_bodies > SG_BODY_CAPACITY) return fail(SG_ERR_CAPACITY, "too many scene bodies");
    if (frame->n_bodies && !frame->bodies) return fail(SG_ERR_INVALID, "frame->bodies is NULL");
    if (frame->globals->ground_north[3] != 0.0f)
        return fail(SG_ERR_INVALID,
                    "frames with a local landscape need a context (terrain and primitives): use sg_closest_hit");
    if (n > SG_NOALLOC_MAX_RAYS) return fail(SG_ERR_CAPACITY, "n exceeds SG_NOALLOC_MAX_RAYS rays per call");
    if (n == 0) return SG_OK;
    if (!rays || !hits) return fail(SG_ERR_INVALID, "rays or hits is NULL");
    DeviceGuard guard(device);
    unsigned char *base = nullptr;
    const int status = scratch_address(device, &base);
    if (status != SG_OK) return status;
    sg_sphere *d_bodies = reinterpret_cast<sg_sphere *>(base + kBodiesOffset);
    sg_ray *d_rays = reinterpret_cast<sg_ray *>(base + kRaysOffset);
    sg_hit *d_hits = reinterpret_cast<sg_hit *>(base + kHitsOffset);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
    // closest_hit (pathtrace.wgsl:173-185) reads the bodies, their count and
    // the globals only; a landscape-free frame needs nothing else.
    sg::TraceParams p;
    std::memset(&p, 0, sizeof(p));
    p.s.g = *frame->globals;
    p.s.counts[0] = frame->n_bodies;
    p.bodies = reinterpret_cast<const float4 *>(d_bodies);
    p.table_stride = SG_RING_TABLE_MAX_BINS;
    if (frame->n_bodies) {
        e = cudaMemcpyAsync(d_bodies, frame->bodies, frame->n_bodies * sizeof(sg_sphere), cudaMemcpyHostToDevice,
                            stream);
        if (e != cudaSuccess) return cuda_fail(e, "copying the bodies");
    }
    e = cudaMemcpyAsync(d_rays, rays, (size_t)n * sizeof(sg_ray), cudaMemcpyHostToDevice, stream);
    if (e != cudaSuccess) return cuda_fail(e, "copying the rays");
    e = sg::launch_closest_hit(p, d_rays, d_hits, n, stream);
    if (e != cudaSuccess) return cuda_fail(e, "closest_hit launch");
    e = cudaMemcpyAsync(hits, d_hits, (size_t)n * sizeof(sg_hit), cudaMemcpyDeviceToHost, stream);
    if (e != cudaSuccess) return cuda_fail(e, "copying the hits");
    e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
    return SG_OK;
}
