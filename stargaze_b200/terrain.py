"""Heightfield and prop data in the reference's landscape layouts.

Terrain layout (src/terrain.rs:781-838, src/shaders/terrain.wgsl:1-20): for a
grid of `cells` cells per side (a power of two, leaves of 2x2 cells),
`V = (cells + 1)^2` vertices and `N = (4 L^2 - 1) / 3` quadtree nodes
(`L = cells / 2` leaves per side):

    heights[V] | dx[V], dz[V] (only when cells <= 1024) | (min, max)[N]

Nodes are in breadth-first heap order: node `n` has children `4n + 1 + c`,
child `c` covering `(x + (c & 1) * size/2, z + (c >> 1) * size/2)`; within a
level that is Morton order. The device appends the node AABBs and vertex
cache that `cache_terrain_geometry` computes.

Props (ground.wgsl:3-12, :167-240): a flat list of primitives in which a
group marker (`center.w < 0`) bounds the next `-center.w` entries. Nesting
markers makes the list a stackless depth-first BVH that the reference's own
traversal loop walks; `build_prop_bvh` builds one over any number of props.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi

EXTENT = 16_000.0  # terrain half extent at scale 1 (src/terrain.rs:13)


def terrain_scale(radius_m: float) -> float:
    """terrain_scale (terrain.wgsl:25-27)."""
    return float(np.clip(np.float32(radius_m) / np.float32(200000.0), np.float32(0.0001), np.float32(1.0)))


def coordinates(cells: int, scale: float = 1.0) -> np.ndarray:
    """terrain_coordinate (terrain.wgsl:28-31) in f32 for i = 0..cells."""
    i = np.arange(cells + 1, dtype=np.float32)
    u = np.float32(2.0) * i / np.float32(cells) - np.float32(1.0)
    return (u * np.abs(u) * np.float32(16000.0) * np.float32(scale)).astype(np.float32)


def node_count(cells: int) -> int:
    leaves = cells // 2
    return (4 * leaves * leaves - 1) // 3


def bounds_offset(cells: int) -> int:
    return (cells + 1) ** 2 * (1 if cells > 1024 else 3)


def terrain_floats(cells: int) -> int:
    """Floats of the full device layout including the cache."""
    v = (cells + 1) ** 2
    n = node_count(cells)
    return bounds_offset(cells) + 2 * n + 6 * n + v * (2 if cells > 1024 else 6)


def _lattice(ix: np.ndarray, iz: np.ndarray, octave: int, seed: int) -> np.ndarray:
    """Uniform [0, 1) lattice values from a 64-bit integer hash."""
    h = (ix.astype(np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ (iz.astype(np.uint64) * np.uint64(0xC2B2AE3D27D4EB4F))
    h ^= np.uint64((seed * 0x165667B19E3779F9 + octave * 0x27D4EB2F165667C5) & 0xFFFFFFFFFFFFFFFF)
    h ^= h >> np.uint64(33)
    h *= np.uint64(0xFF51AFD7ED558CCD)
    h ^= h >> np.uint64(33)
    h *= np.uint64(0xC4CEB9FE1A85EC53)
    h ^= h >> np.uint64(33)
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def fbm_heights(cells: int, seed: int = 0, octaves: int = 8, amplitude: float = 300.0,
                wavelength: float = 6000.0) -> np.ndarray:
    """Seeded 2-D value-noise fBm (lacunarity 2, gain 0.5) sampled at the
    terrain vertex coordinates, in metres, normalised so that the octave sum
    spans +-amplitude."""
    c = coordinates(cells).astype(np.float64)
    total = np.zeros((cells + 1, cells + 1), dtype=np.float64)
    norm = 0.0
    amp, freq = 1.0, 1.0 / wavelength
    for octave in range(octaves):
        # The grid is separable: lattice cell and weight per column / row,
        # lattice values once on the small lattice, then gathered.
        p = c * freq + 1000.0
        i = np.floor(p).astype(np.int64)
        f = p - i
        u = f * f * (3 - 2 * f)
        i0 = int(i.min())
        span = int(i.max()) - i0 + 2
        lx, lz = np.meshgrid(np.arange(span) + i0, np.arange(span) + i0)
        lattice = _lattice(lx, lz, octave, seed)  # [z, x]
        k = i - i0
        a = lattice[k[:, None], k[None, :]]
        b = lattice[k[:, None], k[None, :] + 1]
        cc = lattice[k[:, None] + 1, k[None, :]]
        d = lattice[k[:, None] + 1, k[None, :] + 1]
        ux, uz = u[None, :], u[:, None]
        value = (a * (1 - ux) + b * ux) * (1 - uz) + (cc * (1 - ux) + d * ux) * uz
        total += amp * (2.0 * value - 1.0)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return (total / norm * amplitude).astype(np.float32).reshape(-1)


def _part1by1(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0xFFFF)
    v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
    v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
    v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
    v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
    return v


def pack_terrain(heights: np.ndarray, cells: int) -> np.ndarray:
    """The `Terrain::data` vector of src/terrain.rs:781-838 for `heights`."""
    if cells < 2 or cells & (cells - 1):
        raise ValueError("cells must be a power of two >= 2")
    width = cells + 1
    h = np.asarray(heights, dtype=np.float32).reshape(width, width)
    offset = bounds_offset(cells)
    n = node_count(cells)
    data = np.zeros(offset + 2 * n, dtype=np.float32)
    data[: width * width] = h.reshape(-1)
    if cells <= 1024:
        c = coordinates(cells)
        idx = np.arange(width)
        lo, hi = np.maximum(idx - 1, 0), np.minimum(idx + 1, cells)
        dx = (h[:, hi] - h[:, lo]) / (c[hi] - c[lo])[None, :]
        dz = (h[hi, :] - h[lo, :]) / (c[hi] - c[lo])[:, None]
        data[width * width: 2 * width * width] = dx.astype(np.float32).reshape(-1)
        data[2 * width * width: 3 * width * width] = dz.astype(np.float32).reshape(-1)
    # Leaves: min/max over the 3x3 vertices of each 2x2-cell leaf.
    leaves = cells // 2
    views = [h[dz: dz + 2 * leaves: 2, dx: dx + 2 * leaves: 2] for dz in range(3) for dx in range(3)]
    lo_grid = np.minimum.reduce(views)
    hi_grid = np.maximum.reduce(views)
    levels = []
    while True:
        levels.append((lo_grid, hi_grid))
        if lo_grid.shape[0] == 1:
            break
        s = lo_grid.shape[0] // 2
        lo_grid = lo_grid.reshape(s, 2, s, 2).min(axis=(1, 3))
        hi_grid = hi_grid.reshape(s, 2, s, 2).max(axis=(1, 3))
    levels.reverse()  # root first
    for level, (lo_g, hi_g) in enumerate(levels):
        size = lo_g.shape[0]
        zi, xi = np.meshgrid(np.arange(size), np.arange(size), indexing="ij")
        morton = (_part1by1(xi) | (_part1by1(zi) << np.uint64(1))).astype(np.int64)
        base = ((4 ** level) - 1) // 3
        heap = base + morton
        data[offset + 2 * heap] = lo_g
        data[offset + 2 * heap + 1] = hi_g
    return data


def height_at(heights: np.ndarray, cells: int, x: float, z: float, radius_m: float) -> float:
    """Surface-frame height (metres, curvature included) of the triangulated
    heightfield at (x, z), bilinear within the cell."""
    scale = terrain_scale(radius_m)
    c = coordinates(cells, scale).astype(np.float64)
    width = cells + 1
    h = np.asarray(heights).reshape(width, width)  # the four corners are widened to f64 below
    ix = int(np.clip(np.searchsorted(c, x) - 1, 0, cells - 1))
    iz = int(np.clip(np.searchsorted(c, z) - 1, 0, cells - 1))
    u = float(np.clip((x - c[ix]) / (c[ix + 1] - c[ix]), 0.0, 1.0))
    v = float(np.clip((z - c[iz]) / (c[iz + 1] - c[iz]), 0.0, 1.0))
    h00, h01 = float(h[iz, ix]), float(h[iz, ix + 1])
    h10, h11 = float(h[iz + 1, ix]), float(h[iz + 1, ix + 1])
    y = (h00 * (1 - u) + h01 * u) * (1 - v) + (h10 * (1 - u) + h11 * u) * v
    r = radius_m
    d2 = x * x + z * z
    return y * scale - d2 / (r + math.sqrt(max(r * r - d2, 0.0)))


def primitive(center, kind: float, extent, yaw: float, albedo, material: float) -> abi.Primitive:
    p = abi.Primitive()
    p.center[:] = [float(center[0]), float(center[1]), float(center[2]), float(kind)]
    p.extent[:] = [float(extent[0]), float(extent[1]), float(extent[2]), float(yaw)]
    p.albedo[:] = [float(albedo[0]), float(albedo[1]), float(albedo[2]), float(material)]
    return p


def _bounds(p: abi.Primitive) -> tuple[np.ndarray, np.ndarray]:
    c = np.array(p.center[:3], np.float64)
    e = np.array(p.extent[:3], np.float64)
    if p.center[3] == 2.25:  # tumbled rock: any orientation
        r = float(np.linalg.norm(e))
        half = np.array([r, r, r])
    else:  # rotate_north: rotation in the east-up plane
        cs, sn = abs(math.cos(p.extent[3])), abs(math.sin(p.extent[3]))
        half = np.array([cs * e[0] + sn * e[1], sn * e[0] + cs * e[1], e[2]])
    return c - half, c + half


def build_prop_bvh(props: list[abi.Primitive], leaf_size: int = 4) -> list[abi.Primitive]:
    """Nested group markers over `props` (median split on the longest axis).

    A marker's box is the union of its subtree, padded by 1 mm relative to
    f32 rounding; `-center.w` counts every following entry of the subtree.
    """
    boxes = [_bounds(p) for p in props]
    out: list[abi.Primitive] = []

    def emit(indices: list[int]) -> None:
        lo = np.min([boxes[i][0] for i in indices], axis=0)
        hi = np.max([boxes[i][1] for i in indices], axis=0)
        if len(indices) <= leaf_size:
            groups = [indices]
        else:
            axis = int(np.argmax(hi - lo))
            order = sorted(indices, key=lambda i: boxes[i][0][axis] + boxes[i][1][axis])
            mid = len(order) // 2
            groups = [order[:mid], order[mid:]]
        marker_at = len(out)
        centre = (lo + hi) * 0.5
        half = (hi - lo) * 0.5 + 1e-3 + 1e-6 * np.abs(centre)
        out.append(primitive(centre, -1.0, half, 0.0, (0, 0, 0), 0.0))
        if len(groups) == 1:
            for i in indices:
                out.append(props[i])
        else:
            for g in groups:
                emit(g)
        out[marker_at].center[3] = -float(len(out) - marker_at - 1)

    if props:
        emit(list(range(len(props))))
    return out


def elevation_pyramid(level: np.ndarray) -> np.ndarray:
    """An area-averaged mip pyramid of a square elevation grid, odd edges
    repeating their last sample (src/volcano.rs:73-93), levels concatenated
    down to 1 x 1."""
    level = np.asarray(level, np.float32)
    width = level.shape[0]
    out = [level.ravel()]
    while width > 1:
        nxt = (width + 1) // 2
        i = np.arange(nxt)
        x0, x1 = 2 * i, np.minimum(2 * i + 1, width - 1)
        level = (np.float32(0.25) * (level[x0][:, x0] + level[x0][:, x1] + level[x1][:, x0] + level[x1][:, x1])).astype(np.float32)
        out.append(level.ravel())
        width = nxt
    return np.concatenate(out)


def volcano_atlas(maps, sites) -> np.ndarray:
    """The measured-elevation atlas of basalt ground in the layout
    `volcano.wgsl` reads (src/volcano.rs:36-96): four map descriptors
    (offset, width, spacing, north offset), nine site records (x, z, cos and
    sin of the site's turn; scale, map, 0, 0) — the first the identity on map
    0 — then each map's pyramid. `maps`: four (elevations (w, w), spacing,
    north offset); `sites`: up to eight (x, z, turn radians, scale, map)."""
    header = np.zeros(4 * 4 + 9 * 8, np.float32)
    header[16:24] = [0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0]
    for i, (x, z, turn, scale, m) in enumerate(sites):
        header[24 + 8 * i:32 + 8 * i] = [x, z, np.cos(turn), np.sin(turn), scale, float(m), 0.0, 0.0]
    parts = [header]
    offset = header.size
    for k, (grid, spacing, north) in enumerate(maps):
        grid = np.asarray(grid, np.float32)
        header[4 * k:4 * k + 4] = [float(offset), float(grid.shape[0]), spacing, north]
        pyramid = elevation_pyramid(grid)
        parts.append(pyramid)
        offset += pyramid.size
    return np.concatenate(parts).astype(np.float32)
