"""The camera-only sky backdrop: the procedural star catalogue binned into the
spherical grid the miss shader walks, and the Milky Way haze panorama.

Restates, for upload through sg_upload_catalogue / sg_upload_milky_way,
* `stars::generate`, `stars::radiance` and `stars::ray_catalogue`
  (src/stars.rs:14-201): 3500 uniform stars plus 2500 along the galactic
  band (the app's `stars::generate(3500, 2500, 0x5EED_1234)`,
  src/headless.rs:165), each a disc of fixed angular radius whose radiance
  spreads a Sirius-scaled irradiance over the disc, binned into a 256 x 128
  longitude-colatitude grid that includes the wraparound seam and poles;
* `sky::panorama` (src/sky.rs:9-119): a 1024 x 512 linear RGB10 haze map
  from lattice value noise.

The reference computes these in f32 on the CPU with Rust's libm; here numpy
does the same steps, so individual values can differ from the reference's
by float rounding. The device shades whatever tables it is given: parity
with the oracle is on the same uploaded tables.
"""
from __future__ import annotations

import math

import numpy as np

f32 = np.float32
GRID_W, GRID_H = 256, 128
PANORAMA_W, PANORAMA_H = 1024, 512
POINT_SOURCE_GAIN = f32(100.0)
BRIGHTEST_STAR_IRRADIANCE = f32(6.4e-10) * POINT_SOURCE_GAIN
GALACTIC_POLE = (0.35, 0.82, 0.45)


class _Rng:
    """xorshift64* (src/stars.rs:14-31)."""

    def __init__(self, seed: int):
        self.state = (seed | 1) & 0xFFFFFFFFFFFFFFFF

    def u32(self) -> int:
        x = self.state
        x ^= x >> 12
        x ^= (x << 25) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 27
        self.state = x
        return ((x * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF) >> 32

    def f32(self) -> np.float32:
        return f32(f32(self.u32()) / f32(4294967295.0))


def _srgb_to_linear(c):
    c = min(max(f32(c), f32(0.0)), f32(1.0))
    if c <= f32(0.04045):
        return f32(c / f32(12.92))
    return f32(f32((c + f32(0.055)) / f32(1.055)) ** f32(2.4))


def blackbody_linear(temp_k) -> list:
    """Tanner Helland's blackbody approximation in linear RGB
    (src/stars.rs:34-58)."""
    t = min(max(f32(temp_k) / f32(100.0), f32(10.0)), f32(400.0))
    r = f32(255.0) if t <= 66.0 else f32(329.69873) * f32(f32(t - 60.0) ** f32(-0.13320476))
    g = (f32(99.4708) * f32(np.log(t)) - f32(161.11957)) if t <= 66.0 else \
        f32(288.12217) * f32(f32(t - 60.0) ** f32(-0.07551485))
    if t >= 66.0:
        b = f32(255.0)
    elif t <= 19.0:
        b = f32(0.0)
    else:
        b = f32(138.51773) * f32(np.log(f32(t - 10.0))) - f32(305.0448)
    return [_srgb_to_linear(f32(v) / f32(255.0)) for v in (r, g, b)]


def _random_dir(rng: _Rng):
    z = f32(1.0) - f32(2.0) * rng.f32()
    phi = f32(2.0 * math.pi) * rng.f32()
    r = f32(np.sqrt(max(f32(1.0) - z * z, f32(0.0))))
    return [f32(r * f32(np.cos(phi))), f32(r * f32(np.sin(phi))), z]


def _star(rng: _Rng, dim):
    u = rng.f32()
    bright = (f32(0.02) + u * u * u * f32(1.6)) * f32(dim)
    temp = f32(2500.0) + f32(12000.0) * rng.f32() ** 2
    angular_radius = min(max(f32(0.7) + f32(2.6) * f32(np.sqrt(bright)), f32(0.7)), f32(3.4)) * f32(0.0004)
    return {"dir": _random_dir(rng), "color": blackbody_linear(temp), "angular_radius": f32(angular_radius),
            "bright": f32(bright)}


def _orthonormal(n):
    """Any unit vector orthogonal to unit `n` (Duff et al. 2017, the basis
    src/stars.rs:99 and the miss shader use)."""
    sign = 1.0 if n[2] >= 0.0 else -1.0
    a = -1.0 / (sign + n[2])
    b = n[0] * n[1] * a
    return np.array([b, sign + n[1] * n[1] * a, -n[1]])


def generate(count: int = 3500, band: int = 2500, seed: int = 0x5EED1234) -> list:
    """`stars::generate` (src/stars.rs:91-119)."""
    rng = _Rng(seed)
    out = [_star(rng, 1.0) for _ in range(count)]
    n = np.array(GALACTIC_POLE, np.float32)
    n = (n / np.linalg.norm(n)).astype(np.float32)
    u = _orthonormal(n).astype(np.float32)
    v = np.cross(n, u).astype(np.float32)
    v = (v / np.linalg.norm(v)).astype(np.float32)
    for _ in range(band):
        a = f32(2.0 * math.pi) * rng.f32()
        spread = (rng.f32() + rng.f32() + rng.f32() - f32(1.5)) * f32(0.28)
        d = (u * f32(np.cos(a)) + v * f32(np.sin(a)) + n * spread).astype(np.float32)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        s = _star(rng, 0.28)
        s["dir"] = [f32(x) for x in d]
        s["color"] = blackbody_linear(f32(2500.0) + f32(6000.0) * rng.f32())
        out.append(s)
    return out


def radiance(star) -> list:
    """`stars::radiance` (src/stars.rs:134-139)."""
    radius = f32(min(max(float(star["angular_radius"]), 1e-6), 0.1))
    irradiance = BRIGHTEST_STAR_IRRADIANCE * star["bright"] / f32(1.62)
    rad = irradiance / (f32(math.pi) * radius * radius)
    return [f32(c * rad) for c in star["color"]]


def ray_catalogue(stars: list) -> tuple[np.ndarray, np.ndarray]:
    """`stars::ray_catalogue` (src/stars.rs:152-201): (n, 8) float32 rows of
    (direction xyz, sin^2 of the angular radius, radiance rgb, 0) and the
    u32 cell table: 32,769 offsets into the index list that follows them."""
    cells = [[] for _ in range(GRID_W * GRID_H)]
    data = np.zeros((max(len(stars), 1), 8), np.float32)
    cell_phi = (np.arange(GRID_W) + 0.5) * (2.0 * math.pi) / GRID_W
    for index, star in enumerate(stars):
        d = np.array([float(x) for x in star["dir"]], np.float64)
        d /= np.linalg.norm(d)
        radius = min(max(float(star["angular_radius"]), 1e-6), 0.1)
        data[index, :3] = d
        data[index, 3] = math.sin(radius) ** 2
        data[index, 4:7] = radiance(star)
        theta = math.acos(min(max(d[2], -1.0), 1.0))
        phi = math.atan2(d[1], d[0]) + math.pi
        y0 = min(int(max(theta - radius, 0.0) / math.pi * GRID_H), GRID_H - 1)
        y1 = min(int(min(theta + radius, math.pi) / math.pi * GRID_H), GRID_H - 1)
        if theta <= radius or theta + radius >= math.pi:
            lon_radius = math.pi
        else:
            lon_radius = math.asin(min(max(math.sin(radius) / math.sin(theta), 0.0), 1.0))
        sep = np.abs(np.mod(cell_phi - phi + math.pi, 2.0 * math.pi) - math.pi)
        for x in np.nonzero(sep <= lon_radius + math.pi / GRID_W + 1e-6)[0]:
            for y in range(y0, y1 + 1):
                cells[y * GRID_W + int(x)].append(index)
    offsets = np.zeros(GRID_W * GRID_H + 1, np.uint32)
    offsets[1:] = np.cumsum([len(c) for c in cells])
    indices = np.array([i for c in cells for i in c], np.uint32)
    return data, np.concatenate([offsets, indices]).astype(np.uint32)


# --- Milky Way panorama (src/sky.rs) ---------------------------------------

def _lattice(x, y, z):
    m = np.uint64(0xFFFFFFFF)
    u = np.uint64
    x = np.asarray(x).astype(np.int64).astype(np.uint64) & m
    y = np.asarray(y).astype(np.int64).astype(np.uint64) & m
    z = np.asarray(z).astype(np.int64).astype(np.uint64) & m
    h = ((x * u(0x8DA6B343)) ^ (y * u(0xD8163841)) ^ (z * u(0xCB1AB31F)) ^ u(0x5EED1234)) & m
    h = ((h ^ (h >> u(16))) * u(0x7FEB352D)) & m
    h = ((h ^ (h >> u(15))) * u(0x846CA68B)) & m
    return (((h ^ (h >> u(16))) >> u(8)).astype(np.float32) / f32(16777216.0)).astype(np.float32)


def _noise(p):
    """Quintic value noise (src/sky.rs:21-42); p is (..., 3) float32."""
    fl = np.floor(p)
    c = fl.astype(np.int64)
    t = (p - fl).astype(np.float32)
    t = t * t * t * (t * (t * f32(6.0) - f32(15.0)) + f32(10.0))

    def mix(a, b, s):
        return a + (b - a) * s

    def plane(z):
        return mix(mix(_lattice(c[..., 0], c[..., 1], z), _lattice(c[..., 0] + 1, c[..., 1], z), t[..., 0]),
                   mix(_lattice(c[..., 0], c[..., 1] + 1, z), _lattice(c[..., 0] + 1, c[..., 1] + 1, z), t[..., 0]),
                   t[..., 1])
    return mix(plane(c[..., 2]), plane(c[..., 2] + 1), t[..., 2]).astype(np.float32)


def _clouds(p):
    total = np.zeros(p.shape[:-1], np.float32)
    weight = f32(0.53333336)
    for _ in range(4):
        total = total + weight * _noise(p)
        p = (p * f32(2.07) + np.array([13.1, 7.7, 3.3], np.float32)).astype(np.float32)
        weight = weight * f32(0.5)
    return total


def haze_color(longitude, latitude) -> np.ndarray:
    """`sky::color` (src/sky.rs:57-100) for arrays of galactic longitude and
    latitude: (..., 3) linear RGB in [0, 1]."""
    lon = np.asarray(longitude, np.float32)
    lat = np.asarray(latitude, np.float32)
    lon, lat = np.broadcast_arrays(lon, lat)
    tau = f32(2.0 * math.pi)
    lon = (np.mod(lon + f32(math.pi), tau) - f32(math.pi)).astype(np.float32)
    sl, cl = np.sin(lon).astype(np.float32), np.cos(lon).astype(np.float32)
    sb, cb = np.sin(lat).astype(np.float32), np.cos(lat).astype(np.float32)
    direction = np.stack([cl * cb, sl * cb, sb], -1).astype(np.float32)
    equator = np.stack([cl, sl, np.zeros_like(cl)], -1)
    coarse = _noise(equator * f32(3.7) + f32(17.0))
    center = np.exp(f32(-0.5) * (lon / f32(0.72)) ** 2).astype(np.float32)
    midline = f32(0.075) * np.sin(f32(2.0) * lon) + f32(0.10) * (coarse - f32(0.5))
    width = f32(0.12) + f32(0.12) * coarse + f32(0.16) * center
    d5 = direction * f32(5.0)
    warp = np.stack([_noise(d5 + np.array([11.0, 0.0, 0.0], np.float32)),
                     _noise(d5 + np.array([0.0, 19.0, 0.0], np.float32)),
                     _noise(d5 + np.array([0.0, 0.0, 23.0], np.float32))], -1) - f32(0.5)
    clumps = _clouds(direction * f32(10.0) + warp * f32(4.0))
    wisps = _clouds(direction * f32(29.0) + warp * f32(7.0))
    irregular = lat - midline + f32(0.15) * (clumps - f32(0.5))
    band = np.exp(f32(-0.5) * (irregular / width) ** 2)
    halo = f32(0.07) * np.exp(f32(-0.5) * (lat / (width * f32(1.7))) ** 2)
    bulge = f32(0.46) * center * np.exp(f32(-0.5) * ((lat + f32(0.04)) / f32(0.28)) ** 2)
    starlight = band * (f32(0.05) + f32(1.35) * clumps ** 2) * (f32(0.60) + f32(0.70) * wisps) + bulge
    spine = midline + f32(0.08) * (_noise(direction * f32(8.0)) - f32(0.5))
    rift_width = f32(0.014) + f32(0.042) * _noise(direction * f32(12.0))
    rift = np.exp(f32(-0.5) * ((lat - spine) / rift_width) ** 2)
    branch_spine = spine + f32(0.13) * np.sin(f32(3.0) * lon + f32(0.7))
    branch = np.exp(f32(-0.5) * ((lat - branch_spine) / f32(0.025)) ** 2)
    dust_clouds = _clouds(direction * f32(19.0) + warp * f32(8.0) + f32(11.0))
    patches = np.clip((f32(0.62) - dust_clouds) * f32(3.0), 0.0, 1.0)
    dust = np.clip(f32(0.82) * rift + f32(0.35) * branch * center + f32(0.65) * patches * band, 0.0, 0.96)
    warmth = np.clip(center * f32(0.85) + (coarse - f32(0.5)) * f32(0.35), 0.0, 1.0)[..., None]
    tint = np.array([0.38, 0.55, 1.0], np.float32) + (np.array([1.0, 0.67, 0.36], np.float32) -
                                                      np.array([0.38, 0.55, 1.0], np.float32)) * warmth
    violet = np.array([0.64, 0.32, 0.85], np.float32) * (halo * (f32(0.5) + clumps))[..., None]
    nebula = np.array([0.85, 0.22, 0.38], np.float32) * (
        band * np.maximum((wisps - f32(0.58)) * f32(2.0), 0.0) * (f32(0.3) + center))[..., None]
    rgb = (tint * starlight[..., None] + nebula) * (f32(1.0) - dust)[..., None] + violet
    rgb = np.clip(rgb, 0.0, 1.0).astype(np.float32)
    rgb[np.abs(lat) > f32(1.35)] = 0.0
    return rgb


def panorama() -> np.ndarray:
    """`sky::panorama` (src/sky.rs:103-119): (512, 1024) u32 texels of
    10-bit linear RGB (r | g << 10 | b << 20)."""
    y = np.arange(PANORAMA_H, dtype=np.float32)
    x = np.arange(PANORAMA_W, dtype=np.float32)
    lat = f32(math.pi) * (f32(0.5) - (y + f32(0.5)) / f32(PANORAMA_H))
    lon = f32(2.0 * math.pi) * (f32(0.5) - (x + f32(0.5)) / f32(PANORAMA_W))
    rgb = haze_color(lon[None, :], lat[:, None])
    q = np.round(rgb * f32(1023.0)).astype(np.uint32)
    return (q[..., 0] | (q[..., 1] << 10) | (q[..., 2] << 20)).astype(np.uint32)


__all__ = ["generate", "radiance", "ray_catalogue", "haze_color", "panorama", "blackbody_linear"]
