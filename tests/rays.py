"""Seeded deterministic ray sets for hit-id / distance parity.

Each set mixes camera rays over the field of view, rays leaving every
non-emissive body from its surface (the integrator's body-anchored bounce
origins, offset by 2e-6 radii as in pathtrace.wgsl:1536), near-grazing rays
at each body's limb, and rays leaving ring planes. Directions are f32 and
deliberately not exactly unit length.
"""
from __future__ import annotations

import numpy as np

from stargaze_b200 import abi
from stargaze_b200.pathtracer import rays_array
from stargaze_b200.scene import Frame


def _unit(v: np.ndarray) -> np.ndarray:
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def seeded_rays(frame: Frame, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = frame.globals
    tan = g.cam_forward[3]
    aspect = g.viewport[0] / max(g.viewport[1], 1.0)
    parts_off, parts_dir, parts_anchor = [], [], []

    # Camera rays (anchor MISS, origin 0).
    m = n // 4
    ndc = rng.uniform(-1.0, 1.0, size=(m, 2))
    d = np.stack([ndc[:, 0] * tan * aspect, ndc[:, 1] * tan, -np.ones(m)], axis=1)
    parts_off.append(np.zeros((m, 3)))
    parts_dir.append(_unit(d))
    parts_anchor.append(np.full(m, abi.MISS, np.uint32))

    bodies = [i for i, b in enumerate(frame.bodies) if b.emissive < 0.5]
    # Surface rays from each reflecting body.
    m = n // 4
    idx = rng.choice(bodies, size=m) if bodies else np.zeros(0, int)
    normal = _unit(rng.normal(size=(m, 3)))
    radius = np.array([frame.bodies[i].radius for i in idx], np.float64)
    offset = normal * (radius * (1.0 + 2.0e-6))[:, None]
    d = _unit(normal + rng.normal(size=(m, 3)) * 0.9)
    d = np.where((np.sum(d * normal, axis=1) < 0)[:, None], -d, d)
    parts_off.append(offset)
    parts_dir.append(d)
    parts_anchor.append(idx.astype(np.uint32))

    # Grazing camera rays at each body's limb (all bodies).
    m = n // 4
    idx = rng.integers(0, len(frame.bodies), size=m)
    dirs = []
    for k, i in enumerate(idx):
        b = frame.bodies[i]
        c = np.array(b.center, np.float64) + np.array(b.center_low[:3], np.float64)
        dist = np.linalg.norm(c)
        axis = c / dist
        perp = _unit(np.cross(axis, rng.normal(size=3)))
        ang = b.radius / dist * (1.0 + rng.uniform(-1e-3, 1e-3))
        dirs.append(_unit(axis * np.cos(ang) + perp * np.sin(ang)))
    parts_off.append(np.zeros((m, 3)))
    parts_dir.append(np.array(dirs).reshape(m, 3))
    parts_anchor.append(np.full(m, abi.MISS, np.uint32))

    # Rays leaving ring planes (or more surface rays if no ring exists).
    m = n - sum(len(p) for p in parts_dir)
    ringed = [i for i, b in enumerate(frame.bodies) if b.ring_params[0] > b.ring_plane[3] and b.ring_params[1] > 0]
    if ringed:
        idx = rng.choice(ringed, size=m)
        offs, ds = [], []
        for i in idx:
            b = frame.bodies[i]
            pole = np.array(b.ring_plane[:3], np.float64)
            t = _unit(np.cross(pole, rng.normal(size=3)))
            r = b.radius * rng.uniform(b.ring_plane[3], b.ring_params[0])
            side = 1.0 if rng.uniform() < 0.5 else -1.0
            offs.append(t * r + pole * side * b.radius * 2e-6)
            dd = _unit(rng.normal(size=3))
            if np.dot(dd, pole) * side < 0:
                dd = dd - 2 * np.dot(dd, pole) * pole
            ds.append(dd)
        parts_off.append(np.array(offs))
        parts_dir.append(np.array(ds))
        parts_anchor.append(idx.astype(np.uint32))
    else:
        idx = rng.integers(0, len(frame.bodies), size=m)
        parts_off.append(np.zeros((m, 3)))
        parts_dir.append(_unit(rng.normal(size=(m, 3))))
        parts_anchor.append(np.full(m, abi.MISS, np.uint32))

    return rays_array(np.concatenate(parts_off).astype(np.float32), np.concatenate(parts_dir).astype(np.float32),
                      np.concatenate(parts_anchor).astype(np.uint32))


def light_targets(frame: Frame, n: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 1)
    return rng.integers(0, len(frame.bodies), size=n).astype(np.uint32)


def landscape_rays(frame: Frame, heights: np.ndarray, cells: int, n: int, seed: int) -> np.ndarray:
    """Rays leaving the local ground the way landscape_outgoing builds them
    (ground.wgsl:649-662): origins 0.5 cm to 3 m above seeded ground points
    within 200 m, expressed as camera-relative AU offsets (anchor MISS);
    directions spread over the sphere with a bias towards the horizon."""
    from stargaze_b200.terrain import height_at

    rng = np.random.default_rng(seed)
    g = frame.globals
    east = np.array(g.ground_east[:3], np.float64)
    up = np.array(g.ground_up[:3], np.float64)
    north = np.array(g.ground_north[:3], np.float64)
    h = float(g.ground_east[3])
    radius = float(g.ground_up[3])
    metres_per_au = 149597870700.0
    offs, dirs = [], []
    for _ in range(n):
        x, z = rng.uniform(-200.0, 200.0, size=2)
        y = height_at(heights, cells, x, z, radius) + rng.uniform(0.005, 3.0)
        p = np.array([x, y - h, z])
        offs.append((east * p[0] + up * p[1] + north * p[2]) / metres_per_au)
        d = rng.normal(size=3)
        d[1] = d[1] * 0.4 + 0.05
        d /= np.linalg.norm(d)
        dirs.append(east * d[0] + up * d[1] + north * d[2])
    return rays_array(np.array(offs, np.float32), np.array(dirs, np.float32), abi.MISS)
