"""Closest hits on the full terrain workload (4096^2-cell fBm heightfield
under the min/max quadtree, 2,000 rocks and boxes and 5,000 ellipsoids in
the group-marker BVH, one star): 100,000 seeded rays — camera-space rays
over the scene, rays leaving the ground in every direction, rays aimed at
the props — through the CUDA library and the oracle. Hit ids and distances
must be bit-exact and normals within 2e-6, as on the fixture-sized scenes
(test_cuda_parity.py); light visibility toward the star must take the same
0/1 decisions."""
import numpy as np
import pytest

import known_answers as ka
from oracle.binding import OracleTracer
from rays import landscape_rays, seeded_rays
from stargaze_b200 import abi, workloads as W
from stargaze_b200.pathtracer import PathTracer, rays_array

pytestmark = pytest.mark.gpu

METRES_PER_AU = 149597870700.0


def prop_rays(frame, n: int, seed: int) -> np.ndarray:
    """Rays from 1-3 m above the ground 5-60 m from a seeded prop, aimed at
    a jittered point of its box (camera-relative AU offsets, anchor MISS)."""
    rng = np.random.default_rng(seed)
    g = frame.globals
    east, up, north = (np.array(v[:3], np.float64) for v in (g.ground_east, g.ground_up, g.ground_north))
    h = float(g.ground_east[3])
    props = [p for p in frame.ground if p.center[3] >= 0.0]
    offs, dirs = [], []
    for _ in range(n):
        p = props[rng.integers(len(props))]
        c = np.array(p.center[:3], np.float64)
        e = np.array(p.extent[:3], np.float64)
        angle = rng.uniform(0.0, 2.0 * np.pi)
        dist = rng.uniform(5.0, 60.0)
        o = c + np.array([np.cos(angle) * dist, rng.uniform(1.0, 3.0), np.sin(angle) * dist])
        t = c + e * rng.uniform(-0.8, 0.8, 3)
        d = (t - o) / np.linalg.norm(t - o)
        q = o - np.array([0.0, h, 0.0])
        offs.append((east * q[0] + up * q[1] + north * q[2]) / METRES_PER_AU)
        dirs.append(east * d[0] + up * d[1] + north * d[2])
    return rays_array(np.array(offs, np.float32), np.array(dirs, np.float32), abi.MISS)


def test_full_terrain_scene_hits_are_bit_exact():
    wl, land = W.terrain_1080p()
    f = wl.frame
    rays = np.concatenate([seeded_rays(f, 20000, seed=501),
                           landscape_rays(f, land.heights, land.cells, 60000, seed=502),
                           prop_rays(f, 20000, seed=503)])
    gpu = PathTracer((1, 1), ka.test_options())
    cpu = OracleTracer((1, 1), ka.test_options())
    for t in (gpu, cpu):
        t.upload_terrain(land.terrain, land.cells)
    hits, ref = gpu.closest_hit(f, rays), cpu.closest_hit(f, rays)
    idx = ref["index"]
    assert (idx == abi.TERRAIN_ID).mean() > 0.3
    assert ((idx > abi.LOCAL_BASE) & (idx < abi.TERRAIN_ID)).sum() > 5000  # props
    np.testing.assert_array_equal(hits["index"], ref["index"])
    np.testing.assert_array_equal(hits["distance"], ref["distance"])
    hit = idx != abi.MISS
    assert np.abs(hits["normal"][hit] - ref["normal"][hit]).max() < 2e-6
    # Shadow rays from the ground rays' origins toward the star.
    star = next(i for i, b in enumerate(f.bodies) if b.emissive >= 0.5)
    vis_rays = rays[20000:80000].copy()
    s = f.bodies[star]
    c = np.array(s.center[:3], np.float64) + np.array(s.center_low[:3], np.float64)
    d = c[None, :] - vis_rays["offset"].astype(np.float64)
    vis_rays["direction"] = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    lights = np.full(len(vis_rays), star, np.uint32)
    vis, vref = gpu.light_visibility(f, vis_rays, lights), cpu.light_visibility(f, vis_rays, lights)
    assert (vref > 0).sum() > 10000 and (vref == 0).sum() > 100  # lit and shadowed ground
    np.testing.assert_array_equal(vis > 0, vref > 0)
    gpu.close()
