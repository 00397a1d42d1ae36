"""Shared cases of the adjoint tests: scenes, parameter directions and the
finite-difference machinery (common random numbers: every render of a
difference uses the same noise keys).

The adjoint has no reference counterpart (stargaze renders forward only),
so its checks are (1) the oracle's forward-mode tangent against central
differences of the oracle's own forward render, and (2) the CUDA backward
against the oracle tangent and against central differences of the CUDA
forward.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from stargaze_b200 import workloads as W
from stargaze_b200.scene import Frame


@dataclass
class Direction:
    """A direction in parameter space: per-slot table tangents, (bodies, 3)
    ring albedo / body colour tangents, an albedo-map tangent."""

    ring_tau: dict[int, np.ndarray] = field(default_factory=dict)
    ring_albedo: np.ndarray | None = None
    body_color: np.ndarray | None = None
    albedo_map: np.ndarray | None = None

    def oracle_kwargs(self) -> dict:
        return {"ring_tau": self.ring_tau or None, "ring_albedo": self.ring_albedo,
                "body_color": self.body_color, "albedo_map": self.albedo_map}

    def dot(self, grads, absolute: bool = False) -> float:
        """Directional derivative from a PathTracer.backward result (or the
        sum of |gradient * direction| with `absolute`)."""
        f = np.abs if absolute else (lambda a: a)
        total = 0.0
        for slot, t in self.ring_tau.items():
            total += float(f(grads.ring_tau[slot, : t.size].astype(np.float64) * t).sum())
        if self.ring_albedo is not None:
            total += float(f(grads.ring_albedo.astype(np.float64) * self.ring_albedo).sum())
        if self.body_color is not None:
            total += float(f(grads.body_color.astype(np.float64) * self.body_color).sum())
        if self.albedo_map is not None:
            total += float(f(grads.albedo_map.astype(np.float64) * self.albedo_map).sum())
        return total


def apply(frame: Frame, tables: dict, albedo_map, d: Direction, h: float):
    """Frame, ring tables and albedo map moved by h along d."""
    f = frame.copy()
    t = {k: v.copy() for k, v in tables.items()}
    for slot, v in d.ring_tau.items():
        t[slot] = (t[slot] + np.float32(h) * v).astype(np.float32)
    n = len(f.bodies)
    for i in range(n):
        for c in range(3):
            if d.ring_albedo is not None:
                f.bodies[i].ring_color[c] += h * float(d.ring_albedo[i, c])
            if d.body_color is not None:
                f.bodies[i].color[c] += h * float(d.body_color[i, c])
    m = None
    if albedo_map is not None:
        m = albedo_map if d.albedo_map is None else (albedo_map + np.float32(h) * d.albedo_map).astype(np.float32)
    return f, t, m


def ring_scene(width: int, height: int, spp: int) -> W.Workload:
    """The ring-and-eclipse scene (512-bin table, binary star, moon)."""
    return W.rings_1080p(width, height, spp)


def tau_band(wl: W.Workload, lo: int, hi: int) -> Direction:
    """Relative direction over table bins [lo, hi): tangent = tau there."""
    tau = wl.ring_tables[0]
    v = np.zeros_like(tau)
    v[lo:hi] = tau[lo:hi]
    return Direction(ring_tau={0: v})


def body_direction(wl: W.Workload, body: int, relative: bool = True) -> Direction:
    n = len(wl.frame.bodies)
    d = np.zeros((n, 3), np.float32)
    d[body] = wl.frame.bodies[body].color[:3] if relative else 1.0
    return Direction(body_color=d)


def ring_albedo_direction(wl: W.Workload, body: int) -> Direction:
    n = len(wl.frame.bodies)
    d = np.zeros((n, 3), np.float32)
    d[body] = 1.0
    return Direction(ring_albedo=d)


def loss_weights(width: int, height: int, kind: str = "ones") -> np.ndarray:
    """d loss / d image: all ones (total brightness) or a seeded field."""
    if kind == "ones":
        dl = np.ones((width * height, 4), np.float32)
    else:
        dl = np.random.default_rng(5).uniform(0.0, 1.0, (width * height, 4)).astype(np.float32)
    dl[:, 3] = 0.0
    return dl


def terrain_map_scene(width: int, height: int, spp: int, texels: int = 64, extent_m: float = 400.0):
    """A small terrain scene (256 cells, 50 rocks + 100 ellipsoids within
    10-200 m) whose ground albedo comes from a seeded texels^2 map with
    values in [0.05, 0.6] over +-extent_m."""
    wl, land = W.terrain_1080p(width=width, height=height, spp=spp, cells=256, rocks=50, foliage=100,
                               prop_range=(10.0, 200.0))
    rng = np.random.default_rng(17)
    land.albedo_map = rng.uniform(0.05, 0.6, (texels, texels)).astype(np.float32)
    land.map_extent = extent_m
    return wl, land


def map_direction(land, seed: int = 3) -> Direction:
    """A seeded direction over every map texel."""
    v = np.random.default_rng(seed).uniform(-1.0, 1.0, land.albedo_map.shape).astype(np.float32)
    return Direction(albedo_map=v)
