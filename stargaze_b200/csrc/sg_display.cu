// sg_display.cu — the display side of the path tracer without a graphics
// API: automatic exposure metering (exposure.wgsl) and the resolve of the
// linear HDR accumulation into an exposed, ACES-mapped image (display.wgsl),
// written to a device buffer as 8-bit sRGB (the reference's Rgba8UnormSrgb
// swapchain and headless render target) or as linear float.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "sg_internal.h"

namespace sg {

namespace {

constexpr uint32_t kBins = kExposureBins;
constexpr float kLogMin = -24.0f;
constexpr float kLogMax = 24.0f;
constexpr float kMeterFloor = 1.0e-3f;
constexpr float kMinExposure = 1.0e-8f;
constexpr float kMaxExposure = 1.0e8f;

// measure (exposure.wgsl:52-79): a log2 luminance histogram over the central
// half of the viewport (origin = size / 4 on each side). The Milky Way
// backdrop luminance (w) is taken out first. Each CTA bins into shared
// memory and adds its non-empty bins to the global histogram.
__global__ void __launch_bounds__(256) exposure_measure_kernel(const float4 *mean, uint32_t width, uint32_t height,
                                                               uint32_t *histogram) {
    __shared__ uint32_t bins[kBins];
    for (uint32_t k = threadIdx.x; k < kBins; k += blockDim.x) bins[k] = 0u;
    __syncthreads();
    const uint32_t ox = width / 4u, oy = height / 4u;
    const uint32_t mw = width - 2u * ox, mh = height - 2u * oy;
    const uint32_t n = mw * mh;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t x = ox + k % mw, y = oy + k / mw;
        const float4 hdr = mean[y * width + x];
        const float luminance = fmaxf(0.0f, hdr.x * 0.2126f + hdr.y * 0.7152f + hdr.z * 0.0722f - hdr.w);
        float safe = luminance;
        if (!(safe > 0.0f)) safe = exp2f(kLogMin);  // zero and NaN fall into the darkest bin
        safe = fminf(fmaxf(safe, exp2f(kLogMin)), exp2f(kLogMax));
        const float t = (log2f(safe) - kLogMin) / (kLogMax - kLogMin);
        const uint32_t bin = (uint32_t)fminf(fmaxf(t * (float)kBins, 0.0f), (float)(kBins - 1u));
        atomicAdd(&bins[bin], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < kBins; k += blockDim.x)
        if (bins[k] != 0u) atomicAdd(&histogram[k], bins[k]);
}

// resolve (exposure.wgsl:81-109): the percentile bin's luminance, the target
// exposure key / luminance, eased by 15 % per call.
__global__ void exposure_resolve_kernel(const uint32_t *histogram, ExposureState *e) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (e->enabled < 0.5f) return;
    uint32_t total = 0;
    for (uint32_t i = 0; i < kBins; ++i) total += histogram[i];
    if (total == 0u) return;
    const float p = fminf(fmaxf(e->percentile, 0.0f), 1.0f);
    const uint32_t cutoff = max(1u, (uint32_t)ceilf((float)total * p));
    uint32_t cumulative = 0, bin = 0;
    for (uint32_t i = 0; i < kBins; ++i) {
        cumulative += histogram[i];
        if (cumulative >= cutoff) {
            bin = i;
            break;
        }
    }
    const float t = ((float)bin + 0.5f) / (float)kBins;
    const float measured = fmaxf(exp2f(kLogMin + t * (kLogMax - kLogMin)), kMeterFloor);
    const float desired = fminf(fmaxf(e->key / measured, kMinExposure), kMaxExposure);
    e->value = fminf(fmaxf(e->value + (desired - e->value) * 0.15f, kMinExposure), kMaxExposure);
}

__device__ __forceinline__ float4 texel(const float4 *img, int x, int y, int w, int h) {
    x = min(max(x, 0), w - 1);
    y = min(max(y, 0), h - 1);
    return img[(size_t)y * w + x];
}

// WGSL mix(a, b, t) = a * (1 - t) + b * t.
__device__ __forceinline__ float mixw(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float3 bilinear(float4 a, float4 b, float4 c, float4 d, float wx, float wy) {
    return make_float3(mixw(mixw(a.x, b.x, wx), mixw(c.x, d.x, wx), wy), mixw(mixw(a.y, b.y, wx), mixw(c.y, d.y, wx), wy),
                       mixw(mixw(a.z, b.z, wx), mixw(c.z, d.z, wx), wy));
}

__device__ __forceinline__ float aces(float x) {
    return fminf(fmaxf((x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f), 0.0f), 1.0f);
}

// The sRGB transfer function a Rgba8UnormSrgb target applies on write,
// then rounding to 8 bits.
__device__ __forceinline__ uint32_t srgb8(float c) {
    const float s = c <= 0.0031308f ? 12.92f * c : 1.055f * powf(c, 1.0f / 2.4f) - 0.055f;
    return (uint32_t)fminf(fmaxf(s * 255.0f + 0.5f, 0.0f), 255.0f);
}

// fs (display.wgsl:69-97) for every pixel of a `dw` x `dh` target: bilinear
// sample of the trace-resolution accumulation and backdrop at the pixel
// centre, exposure in stops (automatic or manual, plus bias), the backdrop
// as a gain-limited layer, ACES tone curve.
__global__ void __launch_bounds__(256) display_kernel(DisplayParams D) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.out_width * D.out_height) return;
    const uint32_t ox = k % D.out_width, oy = k / D.out_width;
    const int w = (int)D.width, h = (int)D.height;
    // Pixel-centre coordinates rounded step by step (no fused multiply-add),
    // so that the neighbour weights are reproducible: at 1:1 a weight of
    // 1e-6 instead of 0 on a neighbour a million times brighter is visible.
    const float u = __fdiv_rn(__fadd_rn((float)ox, 0.5f), (float)D.out_width);
    const float v = __fdiv_rn(__fadd_rn((float)oy, 0.5f), (float)D.out_height);
    const float px = __fsub_rn(__fmul_rn(u, (float)w), 0.5f), py = __fsub_rn(__fmul_rn(v, (float)h), 0.5f);
    const float fx = floorf(px), fy = floorf(py);
    const int lx = (int)fx, ly = (int)fy;
    const float wx = __fsub_rn(px, fx), wy = __fsub_rn(py, fy);
    const float4 a = texel(D.mean, lx, ly, w, h), b = texel(D.mean, lx + 1, ly, w, h);
    const float4 c = texel(D.mean, lx, ly + 1, w, h), d = texel(D.mean, lx + 1, ly + 1, w, h);
    const float3 hdr = bilinear(a, b, c, d, wx, wy);
    float3 sky = make_float3(0.0f, 0.0f, 0.0f);
    if (D.backdrop) {
        sky = bilinear(texel(D.backdrop, lx, ly, w, h), texel(D.backdrop, lx + 1, ly, w, h),
                       texel(D.backdrop, lx, ly + 1, w, h), texel(D.backdrop, lx + 1, ly + 1, w, h), wx, wy);
    }
    const bool automatic = D.automatic != 0;
    const float base = automatic ? D.state->value : D.manual;
    // Exposure in stops, capped before multiplying so extreme controls stay
    // finite.
    const float stops = fminf(fmaxf(log2f(fminf(fmaxf(base, 1.0e-30f), 1.0e30f)) + fminf(fmaxf(D.bias, -100.0f), 100.0f),
                                    -100.0f),
                              100.0f);
    const float multiplier = exp2f(stops);
    const float backdrop_gain = fminf(multiplier, 0.04f / fmaxf(D.milky_way, 1.0e-30f));
    const float cap = 1.0e6f / multiplier;
    const float x0 = fminf(fmaxf(hdr.x - sky.x, 0.0f), cap) * multiplier + sky.x * backdrop_gain;
    const float x1 = fminf(fmaxf(hdr.y - sky.y, 0.0f), cap) * multiplier + sky.y * backdrop_gain;
    const float x2 = fminf(fmaxf(hdr.z - sky.z, 0.0f), cap) * multiplier + sky.z * backdrop_gain;
    const float r = aces(x0), g = aces(x1), bl = aces(x2);
    if (D.format == SG_DISPLAY_RGBA32F) {
        reinterpret_cast<float4 *>(D.out)[k] = make_float4(r, g, bl, 1.0f);
    } else {
        reinterpret_cast<uint32_t *>(D.out)[k] = srgb8(r) | (srgb8(g) << 8) | (srgb8(bl) << 16) | (255u << 24);
    }
}

}  // namespace

cudaError_t launch_exposure(const float4 *mean, uint32_t width, uint32_t height, uint32_t *histogram,
                            ExposureState *state, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(histogram, 0, kBins * sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    const uint32_t n = (width - 2u * (width / 4u)) * (height - 2u * (height / 4u));
    if (n > 0) {
        const uint32_t blocks = std::min<uint32_t>((n + 255u) / 256u, 1184u);
        exposure_measure_kernel<<<blocks, 256, 0, stream>>>(mean, width, height, histogram);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    exposure_resolve_kernel<<<1, 32, 0, stream>>>(histogram, state);
    return cudaGetLastError();
}

cudaError_t launch_display(const DisplayParams &d, cudaStream_t stream) {
    const uint32_t n = d.out_width * d.out_height;
    if (n == 0) return cudaSuccess;
    display_kernel<<<(n + 255u) / 256u, 256, 0, stream>>>(d);
    return cudaGetLastError();
}

}  // namespace sg
