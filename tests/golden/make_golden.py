"""Generate the golden fixtures under tests/golden/ with the CPU oracle.

    python tests/golden/make_golden.py [image names]

The oracle is itself pinned against the reference's known-answer tests
(tests/test_oracle_known_answers.py); these fixtures freeze its outputs on
seeded inputs so the CUDA library (tests/test_cuda_parity.py) and any later
oracle change (tests/test_golden.py) are checked against the same numbers
on a machine where the oracle is not rebuilt.
"""
from __future__ import annotations

import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from oracle.binding import OracleTracer  # noqa: E402
from rays import landscape_rays, light_targets, seeded_rays  # noqa: E402
import known_answers as ka  # noqa: E402
from stargaze_b200 import abi  # noqa: E402
from stargaze_b200.pathtracer import rays_array  # noqa: E402
from stargaze_b200.scene import body, frame  # noqa: E402
from stargaze_b200.workloads import rings_1080p, spheres_256, terrain_1080p, with_air, with_mottle  # noqa: E402

N_RAYS = 2048


def transport_scene():
    f = frame()
    f.bodies = [
        body([0.0, 0.0, -3.0], 1.0, [0.8] * 3, False),
        body([0.0, 4.0, 2.0], 0.8, [10.0] * 3, True),
        body([0.0, 2.0, 0.0], 0.5, [0.0] * 3, False),
        body([2.0, 0.0, -1.0], 1.0, [0.9] * 3, False),
    ]
    return f, {}


def terrain_small(width=96, height=54):
    """The terrain workload at fixture size: 256 cells, 200 + 500 props
    within 10-200 m of the observer."""
    return terrain_1080p(width=width, height=height, cells=256, rocks=200, foliage=500, prop_range=(10.0, 200.0))


def vegetate(frame):
    """Turn the terrain fixture's foliage ellipsoids into vegetation
    primitives in turn (3 conifer, 4 grass, 5 trunk, 1 ellipsoid); each stays
    inside its box, so the prop BVH's bounds still hold."""
    kinds = [3.0, 4.0, 5.0, 1.0]
    k = 0
    for prim in frame.ground:
        if prim.center[3] == 1.0:
            prim.center[3] = kinds[k % 4]
            k += 1
    return frame


def scenes():
    s = spheres_256()
    r = rings_1080p()
    t, _land = terrain_small()
    v, _land = terrain_small()
    return {
        "transport": transport_scene(),
        "spheres_256": (s.frame, s.ring_tables),
        "rings_1080p": (r.frame, r.ring_tables),
        "shadow_ring": (ka.shadow_ring_scene(), {}),
        "terrain": (t.frame, {}),
        "vegetation": (vegetate(v.frame), {}),
    }


def landscape_of(name):
    """Terrain data a ray scene needs (None for scenes without terrain)."""
    return terrain_small()[1] if name in ("terrain", "vegetation") else None


def visibility_rays(f, rays, seed):
    """Re-aim each ray at a jittered point of a target body's disc."""
    rng = np.random.default_rng(seed + 7)
    lights = light_targets(f, len(rays), seed)
    dirs = np.zeros((len(rays), 3), np.float64)
    for k, (ray, light) in enumerate(zip(rays, lights)):
        b = f.bodies[light]
        c = np.array(b.center, np.float64) + np.array(b.center_low[:3], np.float64)
        if ray["anchor"] != abi.MISS:
            a = f.bodies[ray["anchor"]]
            c = c - (np.array(a.center, np.float64) + np.array(a.center_low[:3], np.float64))
        c = c - ray["offset"].astype(np.float64)
        jitter = rng.normal(size=3)
        jitter *= b.radius * rng.uniform(0.0, 1.3) / np.linalg.norm(jitter)
        d = c + jitter
        dirs[k] = d / np.linalg.norm(d)
    out = rays.copy()
    out["direction"] = dirs.astype(np.float32)
    return out, lights


def make_tracer(f, tables, dims=(1, 1), land=None, **opts):
    t = OracleTracer(dims, ka.test_options(**opts))
    for slot, tau in tables.items():
        t.upload_ring_profile(slot, tau)
    if land is not None:
        t.upload_terrain(land.terrain, land.cells, getattr(land, "detail", None))
    return t


def ray_fixtures():
    out = {}
    for k, (name, (f, tables)) in enumerate(scenes().items()):
        land = landscape_of(name)
        if land is None:
            rays = seeded_rays(f, N_RAYS, seed=100 + k)
        else:
            half = N_RAYS // 2
            rays = np.concatenate([seeded_rays(f, half, seed=100 + k),
                                   landscape_rays(f, land.heights, land.cells, N_RAYS - half, seed=300 + k)])
        t = make_tracer(f, tables, land=land)
        hits = t.closest_hit(f, rays)
        vrays, lights = visibility_rays(f, rays, seed=200 + k)
        vis = t.light_visibility(f, vrays, lights)
        ring_out = np.zeros((len(f.bodies), len(rays), 4), np.float32)
        for i in range(len(f.bodies)):
            ring_out[i] = t.ring_probe(f, rays, i)
        np.savez_compressed(
            HERE / f"rays_{name}.npz",
            rays=rays.view(np.uint8).reshape(len(rays), -1),
            hit_distance=hits["distance"], hit_index=hits["index"], hit_normal=hits["normal"],
            vis_rays=vrays.view(np.uint8).reshape(len(vrays), -1), vis_lights=lights, visibility=vis,
            ring=ring_out,
        )
        out[name] = (int((hits["index"] != abi.MISS).sum()), int((vis > 0).sum()))
    return out


IMAGES = {
    # name: (workload factory, width, height, spp, batches)
    "spheres_64": (spheres_256, 64, 64, 16, 2),
    "rings_96x54": (rings_1080p, 96, 54, 16, 2),
    "terrain_96x54": (None, 96, 54, 16, 2),
    "terrain_air_96x54": (None, 96, 54, 16, 2),
    "styles_96x32": (None, 96, 32, 16, 2),
    "terrain_alpine_96x54": (None, 96, 54, 16, 2),
    "terrain_dunes_96x54": (None, 96, 54, 16, 2),
    "terrain_basalt_96x54": (None, 96, 54, 16, 2),
    "terrain_vegetation_96x54": (None, 96, 54, 16, 2),
    "mottled_96x54": (rings_1080p, 96, 54, 16, 2),
}

# Landscape themes of the terrain images (ground_counts.z low byte).
THEMES = {"alpine": 3, "basalt": 4, "dunes": 5}


def synthetic_volcano_atlas():
    """A basalt elevation atlas of smooth synthetic elevations in the layout
    of src/volcano.rs (the reference's maps are surveys): a 640 m cone on map
    0 around the observer, a 2 m-spaced summit map 250 m north, two more
    islands on maps 2 and 3 placed by site records."""
    from stargaze_b200.terrain import volcano_atlas

    def grid(width, spacing, peak, radius, ripple):
        c = (np.arange(width) - (width - 1) / 2.0) * spacing
        x, z = np.meshgrid(c, c)
        r = np.hypot(x, z)
        h = peak * np.exp(-(r / radius) ** 2) + ripple * (1.0 + np.sin(x / 37.0) * np.cos(z / 53.0))
        return np.maximum(h, 0.0).astype(np.float32)

    maps = [(grid(65, 20.0, 300.0, 350.0, 6.0), 20.0, 0.0),
            (grid(33, 2.0, 40.0, 20.0, 1.5), 2.0, 250.0),
            (grid(49, 25.0, 200.0, 300.0, 4.0), 25.0, 0.0),
            (grid(49, 25.0, 150.0, 250.0, 3.0), 25.0, 0.0)]
    sites = [(2500.0, 1800.0, 0.6, 1.2, 2), (-3000.0, 900.0, -0.4, 0.9, 3)]
    return volcano_atlas(maps, sites)


def image_workload(name):
    factory, w, h, spp, batches = IMAGES[name]
    if name.startswith("styles"):
        # The six procedural surface styles side by side (no landscape).
        return SimpleNamespace(frame=ka.styles_scene(w, h), ring_tables={}, max_bounces=2), None
    if factory is None:
        wl, land = terrain_small(width=w, height=h)
        if "air" in name:
            with_air(wl.frame, 1)
        for theme, code in THEMES.items():
            if theme in name:
                g = wl.frame.globals
                g.ground_counts[2] = (g.ground_counts[2] & ~255) | code
        if "basalt" in name:
            land.detail = synthetic_volcano_atlas()
        if "vegetation" in name:
            vegetate(wl.frame)
        return wl, land
    wl = factory(width=w, height=h)
    if name.startswith("mottled"):
        # The ring workload with the app's mottle on every non-star body.
        with_mottle(wl.frame)
    return wl, None


def image_fixture(name):
    _factory, w, h, spp, batches = IMAGES[name]
    wl, land = image_workload(name)
    t = make_tracer(wl.frame, wl.ring_tables, dims=(w, h), land=land, samples_per_frame=spp,
                    max_bounces=wl.max_bounces)
    for _ in range(batches):
        t.encode(wl.frame)
    return t.read_pixels()


def image_fixtures(names=None):
    out = {}
    for name in names or IMAGES:
        img = image_fixture(name)
        np.savez_compressed(HERE / f"image_{name}.npz", image=img)
        out[name] = float(img[:, :3].mean())
    return out


if __name__ == "__main__":
    # With image names as arguments, only those image fixtures are rebuilt.
    if len(sys.argv) > 1:
        print(image_fixtures(sys.argv[1:]))
    else:
        print(ray_fixtures())
        print(image_fixtures())
