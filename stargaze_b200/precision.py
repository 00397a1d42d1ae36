"""Hit-distance precision of the integrator's two large-magnitude
intersection sites against double precision.

* Host sphere (ground.wgsl:138-158): a camera metres above a planet-sized
  sphere, rays from grazing to nadir. The reference solves the quadratic in
  f32 metres in the surface frame; the FP64 sites (PathTracer.set_fp64_sites)
  solve it in double from the same f32 inputs.
* Ring plane (rings.wgsl:8-34): camera rays at points of a giant's ring,
  whose centre sits 1e-3 AU from the camera and whose ring radius is a few
  1e8 m.

Both compare the device's answer for the SAME f32 rays with the exact
intersection of those rays computed here in numpy float64, so the figures
are the device arithmetic's error alone.
"""
from __future__ import annotations

import numpy as np

from . import abi
from .pathtracer import PathTracer, rays_array
from .scene import AU_M, Frame


def host_sphere_frame(radius_m: float = 6.4e6, height_m: float = 2.0) -> Frame:
    """A landscape frame with the host sphere alone: a camera `height_m`
    above a `radius_m` host (no terrain, no primitives, no star needed)."""
    f32 = np.float32
    up = np.array([0.0, np.sqrt(f32(0.8)), np.sqrt(f32(0.2))], dtype=np.float32)
    north = np.array([0.0, -up[2], up[1]], dtype=np.float32)
    frame = Frame()
    frame.globals.ground_east[:] = [1.0, 0.0, 0.0, height_m]
    frame.globals.ground_up[:] = [float(up[0]), float(up[1]), float(up[2]), radius_m]
    frame.globals.ground_north[:] = [float(north[0]), float(north[1]), float(north[2]), 1.0]
    body = abi.Sphere()
    metre = f32(1.0) / f32(AU_M)
    body.center[:] = [float(v) for v in -up * ((f32(radius_m) + f32(height_m)) * metre)]
    body.radius = float(f32(radius_m) * metre)
    body.color[:] = [0.3, 0.3, 0.3]
    frame.bodies = [body]
    return frame


def host_sphere_rays(frame: Frame, n: int, seed: int = 0):
    """Camera rays below the horizon, from grazing (1e-6 rad past the
    horizon dip) to nadir, log-spaced in depression angle, uniform azimuth.
    Returns the f32 rays, their exact hit distances in metres and their
    angle past the horizon dip."""
    g = frame.globals
    east = np.array(g.ground_east[:3], np.float64)
    up = np.array(g.ground_up[:3], np.float64)
    north = np.array(g.ground_north[:3], np.float64)
    h, r = float(g.ground_east[3]), float(g.ground_up[3])
    rng = np.random.default_rng(seed)
    dip = np.arccos(r / (r + h))
    depression = dip + np.exp(rng.uniform(np.log(1e-6), np.log(np.pi / 2 - dip), n))
    azimuth = rng.uniform(0.0, 2.0 * np.pi, n)
    local = np.stack([np.cos(depression) * np.sin(azimuth), -np.sin(depression),
                      np.cos(depression) * np.cos(azimuth)], axis=1)
    world = (local[:, :1] * east + local[:, 1:2] * up + local[:, 2:] * north).astype(np.float32)
    # The f32 direction in the frame's f32 basis, observer h above the
    # sphere centred at (0, -r, 0) of the surface frame.
    d = world.astype(np.float64)
    d = np.stack([d @ east, d @ up, d @ north], axis=1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    b = d[:, 1] * (r + h)                     # d . (o - c), o - c = (0, r + h, 0)
    c = h * (2.0 * r + h)                     # |o - c|^2 - r^2
    disc = b * b - c
    hit = disc >= 0.0
    t = np.full(n, np.inf)
    t[hit] = c / (-b[hit] + np.sqrt(disc[hit]))
    return rays_array(np.zeros((1, 3), np.float32), world, abi.MISS), t, depression - dip


def _summary(rel: np.ndarray) -> dict:
    return {"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99)), "max": float(rel.max())}


def host_sphere_precision(n: int, fp64: bool, device: int = 0, seed: int = 0) -> dict:
    """Relative and absolute hit-distance error of the host-sphere
    intersection on `n` seeded rays (sg_closest_hit, f32 or FP64 sites)."""
    frame = host_sphere_frame()
    rays, t64, past = host_sphere_rays(frame, n, seed)
    with PathTracer((1, 1), device=device) as tracer:
        tracer.set_fp64_sites(fp64)
        hits = tracer.closest_hit(frame, rays)
    expected = np.isfinite(t64)
    found = expected & (hits["index"] == abi.LOCAL_BASE)
    got = hits["distance"].astype(np.float64) * AU_M
    rel = np.abs(got[found] - t64[found]) / t64[found]
    grazing = past[found] < 1e-3
    return {"rays": int(n), "hits_expected": int(expected.sum()), "hits_found": int(found.sum()),
            "relative_error": _summary(rel),
            "relative_error_within_1mrad_of_horizon": float(rel[grazing].max()) if grazing.any() else None,
            "relative_error_beyond_1mrad": float(rel[~grazing].max()) if (~grazing).any() else None,
            "absolute_error_m_max": float(np.abs(got[found] - t64[found]).max())}


def ring_bodies(frame: Frame) -> list[int]:
    return [i for i, b in enumerate(frame.bodies) if b.ring_params[0] > b.ring_plane[3] and b.ring_params[1] > 0.0]


def ring_rays(frame: Frame, body: int, n: int, seed: int = 0):
    """Camera rays (anchor MISS, origin 0) at seeded points of body `body`'s
    ring annulus, uniform in area. Returns the f32 rays, the exact plane
    distance (AU) and radius (body radii) of those f32 rays, and which of
    them hit the annulus."""
    b = frame.bodies[body]
    centre = np.array(b.center[:], np.float64) + np.array(b.center_low[:3], np.float64)
    radius = float(b.radius)
    pole = np.array(b.ring_plane[:3], np.float32).astype(np.float64)
    inner, outer = float(b.ring_plane[3]), float(b.ring_params[0])
    u = np.cross(pole, [1.0, 0.0, 0.0] if abs(pole[0]) < 0.9 else [0.0, 1.0, 0.0])
    u /= np.linalg.norm(u)
    v = np.cross(pole, u)
    rng = np.random.default_rng(seed)
    rho = np.sqrt(rng.uniform(inner**2, outer**2, n)) * radius
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    target = centre + rho[:, None] * (np.cos(phi)[:, None] * u + np.sin(phi)[:, None] * v)
    d32 = (target / np.linalg.norm(target, axis=1, keepdims=True)).astype(np.float32)
    d = d32.astype(np.float64)
    t = (centre @ pole) / (d @ pole)
    point = d * t[:, None] - centre
    r = np.linalg.norm(point, axis=1) / radius
    inside = (t > 0.0) & (r >= inner) & (r <= outer)
    return rays_array(np.zeros((1, 3), np.float32), d32, abi.MISS), t, r, inside


def ring_plane_precision(frame: Frame, n: int, fp64: bool, tables=None, device: int = 0, seed: int = 0) -> dict:
    """Relative error of the ring-plane distance and of the hit radius
    (sg_ring_probe, f32 or FP64 sites) on `n` seeded camera rays per ringed
    body of `frame`."""
    out = {}
    with PathTracer((1, 1), device=device) as tracer:
        tracer.set_fp64_sites(fp64)
        for slot, tau in (tables or {}).items():
            tracer.upload_ring_profile(slot, tau)
        for body in ring_bodies(frame):
            rays, t64, r64, inside = ring_rays(frame, body, n, seed)
            probe = tracer.ring_probe(frame, rays, body)
            # Rays within float rounding of either edge may fall either side.
            b = frame.bodies[body]
            edge = (np.abs(r64 - b.ring_plane[3]) < 1e-5) | (np.abs(r64 - b.ring_params[0]) < 1e-5)
            hit = probe[:, 3] == 1.0
            use = inside & hit & ~edge
            t_rel = np.abs(probe[use, 0] - t64[use]) / t64[use]
            r_rel = np.abs(probe[use, 1] - r64[use]) / r64[use]
            out[str(body)] = {"rays": int(n), "hits_expected": int((inside & ~edge).sum()),
                              "hits_found": int(use.sum()), "distance_relative_error": _summary(t_rel),
                              "radius_relative_error": _summary(r_rel)}
    return out


__all__ = ["host_sphere_frame", "host_sphere_rays", "host_sphere_precision", "ring_bodies", "ring_rays",
           "ring_plane_precision"]
