"""CPU restatement of the reference's display side — test infrastructure only.

numpy (float64 unless noted) restatements of
* the centre-weighted luminance histogram and the eased automatic exposure
  (src/shaders/exposure.wgsl:52-109; the region of
  src/pathtracer.rs:40-42; the state written at every encode,
  src/pathtracer.rs:883-905, metered at :980-1000), and
* the display fragment shader (src/shaders/display.wgsl:40-97): bilinear
  upscale of the trace-resolution accumulation, exposure in stops, the
  gain-limited Milky Way layer, the ACES curve, and the sRGB encoding that a
  Rgba8UnormSrgb target (src/headless.rs:13) applies on write.

Only the test suite imports it; the library never does.
"""
from __future__ import annotations

import math

import numpy as np

BINS = 256
LOG_MIN, LOG_MAX = -24.0, 24.0
METER_FLOOR = 1.0e-3
MIN_EXPOSURE, MAX_EXPOSURE = 1.0e-8, 1.0e8
LUMA = np.array([0.2126, 0.7152, 0.0722])


def meter_region(width: int, height: int) -> tuple[int, int, int, int]:
    """(x0, y0, w, h) of the metered centre (exposure_meter_size)."""
    ox, oy = width // 4, height // 4
    return ox, oy, width - 2 * ox, height - 2 * oy


def histogram(mean: np.ndarray, width: int, height: int) -> np.ndarray:
    """measure (exposure.wgsl:52-79) over a (height * width, 4) accumulation."""
    img = np.asarray(mean, np.float32).reshape(height, width, 4)
    ox, oy, w, h = meter_region(width, height)
    region = img[oy:oy + h, ox:ox + w].astype(np.float64)
    lum = np.maximum(0.0, region[..., :3] @ LUMA - region[..., 3]).ravel()
    safe = np.where(lum > 0.0, lum, 2.0 ** LOG_MIN)
    safe = np.clip(safe, 2.0 ** LOG_MIN, 2.0 ** LOG_MAX)
    t = (np.log2(safe) - LOG_MIN) / (LOG_MAX - LOG_MIN)
    bins = np.clip(t * BINS, 0.0, BINS - 1).astype(np.int64)
    return np.bincount(bins, minlength=BINS)


def resolve(hist: np.ndarray, value: float, key: float, percentile: float) -> float:
    """resolve (exposure.wgsl:81-109): one easing step of the exposure."""
    total = int(hist.sum())
    if total == 0:
        return value
    cutoff = max(1, math.ceil(total * min(max(percentile, 0.0), 1.0)))
    bin_ = int(np.searchsorted(np.cumsum(hist), cutoff))
    t = (bin_ + 0.5) / BINS
    measured = max(2.0 ** (LOG_MIN + t * (LOG_MAX - LOG_MIN)), METER_FLOOR)
    desired = min(max(key / measured, MIN_EXPOSURE), MAX_EXPOSURE)
    return min(max(value + (desired - value) * 0.15, MIN_EXPOSURE), MAX_EXPOSURE)


def eased_exposure(mean, width, height, start: float, key: float, percentile: float, encodes: int) -> float:
    """The automatic exposure after `encodes` meterings of an unchanging
    accumulation, starting from the manual exposure `start`."""
    hist = histogram(mean, width, height)
    value = start
    for _ in range(encodes):
        value = resolve(hist, value, key, percentile)
    return value


def aces(x):
    x = np.asarray(x, np.float64)
    return np.clip((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0.0, 1.0)


def srgb8(c):
    """Linear [0, 1] to the 8-bit sRGB code a Rgba8UnormSrgb target stores."""
    c = np.asarray(c, np.float64)
    s = np.where(c <= 0.0031308, 12.92 * c, 1.055 * np.power(np.maximum(c, 0.0), 1.0 / 2.4) - 0.055)
    return np.clip(np.floor(s * 255.0 + 0.5), 0, 255).astype(np.uint8)


def display(mean, width: int, height: int, out_width: int, out_height: int, exposure: float, bias: float = 0.0,
            backdrop=None, milky_way: float = 0.0) -> np.ndarray:
    """fs (display.wgsl:69-97) at every pixel of an out_width x out_height
    target: (out_height, out_width, 3) linear ACES-mapped colours."""
    img = np.asarray(mean, np.float32).reshape(height, width, 4)[..., :3].astype(np.float64)
    sky_img = (np.zeros_like(img) if backdrop is None
               else np.asarray(backdrop, np.float32).reshape(height, width, 4)[..., :3].astype(np.float64))
    # Pixel-centre coordinates in f32, one rounding per operation, as the
    # shader computes them: the neighbour weights then match exactly.
    f32 = np.float32
    u = (np.arange(out_width, dtype=f32) + f32(0.5)) / f32(out_width)
    v = (np.arange(out_height, dtype=f32) + f32(0.5)) / f32(out_height)
    px = u * f32(width) - f32(0.5)
    py = v * f32(height) - f32(0.5)
    lx = np.floor(px).astype(np.int64)
    ly = np.floor(py).astype(np.int64)
    wx = (px - np.floor(px)).astype(np.float64)[None, :, None]
    wy = (py - np.floor(py)).astype(np.float64)[:, None, None]

    def at(a, xs, ys):
        return a[np.clip(ys, 0, height - 1)[:, None], np.clip(xs, 0, width - 1)[None, :]]

    def bilinear(a):
        top = at(a, lx, ly) * (1 - wx) + at(a, lx + 1, ly) * wx
        bot = at(a, lx, ly + 1) * (1 - wx) + at(a, lx + 1, ly + 1) * wx
        return top * (1 - wy) + bot * wy

    hdr, sky = bilinear(img), bilinear(sky_img)
    stops = min(max(math.log2(min(max(exposure, 1.0e-30), 1.0e30)) + min(max(bias, -100.0), 100.0), -100.0), 100.0)
    multiplier = 2.0 ** stops
    backdrop_gain = min(multiplier, 0.04 / max(milky_way, 1.0e-30))
    fore = np.maximum(hdr - sky, 0.0)
    x = np.minimum(fore, 1.0e6 / multiplier) * multiplier + sky * backdrop_gain
    return aces(x)
