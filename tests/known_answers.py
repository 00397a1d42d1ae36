"""The reference's known-answer tests, written once for any tracer.

Each scenario restates one of stargaze's GPU tests (file:line cited) and
runs against a `make(dimensions, options)` factory, so the same assertions
pin the CPU oracle (tests/test_oracle_known_answers.py) and the CUDA library
(tests/test_cuda_known_answers.py). Where a reference tolerance cannot hold
for two independent noise sequences, the scenario uses common random numbers
and says so.
"""
from __future__ import annotations

import math

import numpy as np

from stargaze_b200 import abi
from stargaze_b200.pathtracer import rays_array
from stargaze_b200.scene import body, frame, ringed


def test_options(**fields) -> abi.Options:
    """`test_options()` (src/pathtracer_tests.rs:25-30): no Milky Way."""
    o = abi.default_options()
    o.milky_way = 0.0
    for k, v in fields.items():
        setattr(o, k, v)
    return o


def sample(tracer, f, batches: int) -> np.ndarray:
    """`sample()` (src/pathtracer_tests.rs:184-197)."""
    for _ in range(batches):
        tracer.encode(f)
    return tracer.read_pixels()


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:441-600 — gpu_transport
# ---------------------------------------------------------------------------
def transport(make) -> dict:
    tracer = make((1, 1), test_options(samples_per_frame=64, max_bounces=1, exposure=1.0))
    f = frame()
    black = sample(tracer, f, 1)[0]
    assert np.array_equal(black, np.zeros(4, np.float32)), black
    # An unchanged size preserves the image and the history.
    tracer.resize((1, 1))
    assert tracer.samples() == 64
    assert np.array_equal(tracer.read_pixels()[0], black)
    sample(tracer, f, 1)
    assert tracer.samples() == 128

    # Emission, true silhouettes and inside-sphere roots.
    f.bodies = [body([0.0, 0.0, -1.0], 1e-6, [2.0, 3.0, 4.0], True)]
    assert np.array_equal(sample(tracer, f, 1)[0], np.array([2, 3, 4, 0], np.float32))
    f.bodies[0].center[:] = [0.0, 0.0, 0.0]
    f.bodies[0].radius = 1.0
    assert np.array_equal(sample(tracer, f, 1)[0], np.array([2, 3, 4, 0], np.float32))

    f.bodies = [body([0.0, 0.0, -3.0], 1.0, [0.8] * 3, False), body([0.0, 4.0, 2.0], 0.8, [10.0] * 3, True)]
    seq0 = tracer.sequence()
    full = float(sample(tracer, f, 32)[0][0])
    expected = 0.8 * 10.0 * 0.8**2 / 32.0 * math.sqrt(0.5)
    assert abs(full - expected) < expected * 0.03, (full, expected)
    assert tracer.samples() == 2048

    # An occluder behind the emitter cannot shadow it. The reference compares
    # two independent noise sequences to 1e-6, tighter than their Monte Carlo
    # spread (~2e-4 at 2048 spp); with common random numbers the estimates
    # must be identical.
    crn = make((1, 1), test_options(samples_per_frame=64, max_bounces=1, noise_seed=seq0))
    g = f.copy()
    g.bodies.append(body([0.0, 8.0, 6.0], 1.0, [0.0] * 3, False))
    behind = float(sample(crn, g, 32)[0][0])
    assert abs(behind - full) < 1e-6, (behind, full)
    behind_independent = float(sample(tracer, g, 32)[0][0])
    assert abs(behind_independent - full) < full * 0.01

    # Aligned occluder covers the stellar disc.
    f.bodies.append(body([0.0, 2.0, 0.0], 0.5, [0.0] * 3, False))
    umbra = float(sample(tracer, f, 32)[0][0])
    assert umbra < full * 0.001, (umbra, full)
    # Equal angular discs shifted sideways: partial shadow.
    f.bodies[2].center[0] = 0.4
    f.bodies[2].radius = 0.4
    penumbra = float(sample(tracer, f, 32)[0][0])
    assert full * 0.2 < penumbra < full * 0.85, (penumbra, full)
    # Small aligned disc: annular eclipse.
    f.bodies[2].center[0] = 0.0
    f.bodies[2].radius = 0.2
    annular = float(sample(tracer, f, 32)[0][0])
    assert full * 0.6 < annular < full * 0.85, (annular, full)
    # Multiple emitters add.
    f.bodies.pop()
    f.bodies.append(body([0.0, -4.0, 2.0], 0.8, [10.0] * 3, True))
    binary = float(sample(tracer, f, 32)[0][0])
    assert abs(binary / full - 2.0) < 0.05, (binary, full)
    # MIS does not double count emission reached by BSDF paths.
    tracer.update_options(max_bounces=8)
    bounced = float(sample(tracer, f, 128)[0][0])
    assert abs(bounced / binary - 1.0) < 0.05, (bounced, binary)
    # A white reflector adds indirect light to a directly shadowed point.
    f.bodies = [
        body([0.0, 0.0, -3.0], 1.0, [0.8] * 3, False),
        body([0.0, 4.0, 2.0], 0.8, [10.0] * 3, True),
        body([0.0, 2.0, 0.0], 0.5, [0.0] * 3, False),
        body([2.0, 0.0, -1.0], 1.0, [0.9] * 3, False),
    ]
    indirect = float(sample(tracer, f, 128)[0][0])
    assert indirect > 0.0001, indirect
    tracer.update_options(max_bounces=1)
    direct_only = float(sample(tracer, f, 32)[0][0])
    assert direct_only < 1e-6, direct_only
    # Resizing resets the history and allocates a fresh image.
    tracer.resize((3, 2))
    assert tracer.samples() == 0
    f.globals.viewport[0] = 3.0
    f.globals.viewport[1] = 2.0
    assert len(sample(tracer, f, 1)) == 6
    return dict(full=full, umbra=umbra, penumbra=penumbra, annular=annular, binary=binary,
                bounced=bounced, indirect=indirect, direct_only=direct_only)


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:604-642 — gpu_distant_surface
# ---------------------------------------------------------------------------
def distant_surface(make, size: int = 256) -> dict:
    tracer = make((size, size), test_options(samples_per_frame=16, max_bounces=1, exposure=1.0))
    f = frame()
    f.globals.viewport[:] = [float(size), float(size), 1.0, 0.0]
    dark_counts = {}
    for radius in (1e-4, 1e-6, 1e-7):
        f.globals.cam_forward[3] = radius / 10.0 * 1.3
        f.bodies = [body([0.0, 0.0, -10.0], radius, [0.8] * 3, False),
                    body([5.0, 0.0, -5.0], 0.05, [10000.0] * 3, True)]
        pixels = sample(tracer, f, 4).reshape(size, size, 4)
        lo, hi = size * 100 // 256, size * 156 // 256
        dark = int((pixels[lo:hi, lo:hi, 0] < 0.05).sum())
        dark_counts[radius] = dark
        assert dark == 0, (radius, dark)
    return dark_counts


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:201-237 — noise sequence
# ---------------------------------------------------------------------------
def noise_sequence(make) -> None:
    f = frame()
    f.globals.viewport[:] = [32.0, 32.0, 1.0, 1.0]
    f.globals.cam_forward[3] = 0.5
    f.bodies = [body([0.0, 0.0, -3.0], 1.0, [1.0] * 3, True)]

    def new(seed):
        return make((32, 32), test_options(noise_seed=seed, samples_per_frame=1))

    tracer = new(0)
    first = sample(tracer, f, 1)
    f.scene_time = 1.0  # same geometry, fresh accumulation
    reset = sample(tracer, f, 1)
    assert tracer.samples() == 1
    assert not np.array_equal(first, reset)
    same_seed = new(0)
    assert np.array_equal(first, sample(same_seed, f, 1))
    other_seed = new(12345)
    assert not np.array_equal(first, sample(other_seed, f, 1))
    tracer.set_quality(1, 4, 10)
    quality_reset = sample(tracer, f, 1)
    assert tracer.samples() == 1
    assert not np.array_equal(first, quality_reset)
    assert not np.array_equal(reset, quality_reset)


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:241-314 — quality limits, rest and resume
# ---------------------------------------------------------------------------
def quality_limits(make) -> None:
    tracer = make((1, 1), test_options(samples_per_frame=64, max_bounces=1, sample_limit=65, auto_exposure=1))
    f = frame()
    f.bodies = [body([0.0, 0.0, -1.0], 0.1, [2.0, 3.0, 4.0], True)]
    initial = sample(tracer, f, 1)
    assert tracer.samples() == 64
    assert tracer.needs_redraw()
    sample(tracer, f, 1)
    assert tracer.samples() == 65, "last batch must stop exactly at the limit"
    assert tracer.needs_redraw(), "exposure still needs to settle"
    assert np.array_equal(sample(tracer, f, 60), initial)
    assert tracer.samples() == 65
    assert not tracer.needs_redraw(), "a completed still view should sleep"
    tracer.set_quality(8, 1, 32)
    assert tracer.samples() == 65, "lowering the target preserves the better image"
    assert not tracer.needs_redraw()
    sample(tracer, f, 1)
    assert tracer.samples() == 65, "a lower target must not underflow the counter"
    tracer.set_quality(8, 1, 256)
    assert tracer.needs_redraw()
    sample(tracer, f, 1)
    assert tracer.samples() == 73, "a higher target resumes the existing average"
    tracer.set_quality(8, 2, 256)
    assert tracer.samples() == 0, "changing light transport invalidates the image"
    sample(tracer, f, 1)
    assert tracer.samples() == 8
    tracer.set_quality(8, 2, 8)
    sample(tracer, f, 60)
    assert not tracer.needs_redraw()
    f.scene_time += 1.0
    sample(tracer, f, 1)
    assert tracer.samples() == 8
    assert tracer.needs_redraw(), "a changed scene starts refinement again"


# ---------------------------------------------------------------------------
# src/ring_tests.rs:57-135 — gpu_rings_geometry (probe)
# ---------------------------------------------------------------------------
def rings_geometry(make) -> None:
    tracer = make((1, 1), test_options())
    f = frame()
    r = 0.0004
    f.bodies = [ringed([1.8 * r, 0.0, -10.0], r, [0.0, 0.8, 0.6], 0.7), body([0.0, 0.0, -12.0], 0.1, [1.0] * 3, True)]
    ray = rays_array([0, 0, 0], [[0.0, 0.0, -1.0]], abi.MISS)

    def probe():
        p = tracer.ring_probe(f, ray, 0)[0]
        if p[3] == 0.0:
            return np.zeros(4, np.float32)
        vis = tracer.light_visibility(f, ray, [1])[0]
        return np.array([p[0], p[1], p[2], vis], np.float32)

    p = probe()
    expected = math.exp(-0.7 / 0.6)
    assert abs(p[0] - 10.0) < 1e-5 and abs(p[1] - 1.8) < 1e-4, p
    assert abs(p[2] - expected) < 1e-5 and abs(p[3] - expected) < 1e-5, p
    for offset, pole in ((0.5, [0.0, 0.0, 1.0]), (2.6, [0.0, 0.0, 1.0]), (1.8, [0.0, 1.0, 0.0])):
        f.bodies[0] = ringed([offset * r, 0.0, -10.0], r, pole, 0.7)
        assert np.array_equal(probe(), np.zeros(4, np.float32)), (offset, pole)
    f.bodies[0] = ringed([1.8 * r, 0.0, -10.0], r, [0.0, 0.0, 1.0], 0.7)
    f.bodies[1].center[2] = -9.0
    p = probe()
    assert abs(p[3] - 1.0) < 1e-6, p


# ---------------------------------------------------------------------------
# src/ring_tests.rs:137-202 — gpu_rings_transport
# ---------------------------------------------------------------------------
def rings_transport(make) -> None:
    tracer = make((1, 1), test_options(samples_per_frame=64, max_bounces=1, exposure=1.0))
    f = frame()
    f.bodies = [ringed([1.8, 0.0, -5.0], 1.0, [0.0, 0.0, 1.0], 0.7), body([0.0, 0.0, -9.0], 0.5, [1.0] * 3, True)]
    f.bodies[0].ring_color[:] = [0.0, 0.0, 0.0, 0.0]
    for pole, expected in (([0.0, 0.0, 1.0], math.exp(-0.7)), ([0.0, 0.8, 0.6], math.exp(-0.7 / 0.6))):
        f.bodies[0].ring_plane[0:3] = pole
        p = sample(tracer, f, 256)[0]
        assert abs(p[0] - expected) < 0.02, (p, expected)
    f.bodies[0] = ringed([1.8, 0.0, -5.0], 1.0, [0.0, 0.0, 1.0], 0.7)
    for star_z, same_side in ((15.0, True), (-25.0, False)):
        f.bodies[1] = body([10.0, 0.0, star_z], 0.05, [100_000.0] * 3, True)
        mu = 20.0 / math.sqrt(500.0)
        if same_side:
            factor = (1.0 - math.exp(-0.7 * (1.0 + 1.0 / mu))) / (1.0 + mu)
        else:
            factor = (math.exp(-0.7 / mu) - math.exp(-0.7)) / (mu - 1.0)
        solid_angle = 2.0 * math.pi * (0.05**2 / 500.0) / (1.0 + math.sqrt(1.0 - 0.05**2 / 500.0))
        expected = 0.8 * factor / (4.0 * math.pi) * mu * 100_000.0 * solid_angle
        p = sample(tracer, f, 32)[0]
        assert abs(p[0] / expected - 1.0) < 0.02, (p, expected)
        f.bodies.append(body([5.0, 0.0, (star_z - 5.0) * 0.5], 0.5, [0.0] * 3, False))
        dark = sample(tracer, f, 8)[0]
        assert dark[0] < p[0] * 0.001, (dark, p)
        f.bodies.pop()


# ---------------------------------------------------------------------------
# src/ring_tests.rs:352-413 — gpu_rings_conserve_energy
# ---------------------------------------------------------------------------
def rings_conserve_energy(make) -> list:
    tracer = make((1, 1), test_options())
    energies = []
    for albedo in (0.8, 0.88, 1.0):
        for tau in (0.001, 0.1, 0.7, 2.0):
            for mu in (0.05, 0.5, 1.0):
                e = tracer.ring_energy(albedo, tau, mu, 4096)
                assert 0.0 <= e <= 1.0001, (albedo, tau, mu, e)
                energies.append(e)
    return energies


# ---------------------------------------------------------------------------
# src/ring_tests.rs:415-453 — gpu_rings_null_crossings_preserve_mis
# ---------------------------------------------------------------------------
def rings_null_crossings_preserve_mis(make, size: int = 64) -> tuple[float, float]:
    tracer = make((size, size), test_options(samples_per_frame=64, max_bounces=1))
    f = frame()
    f.globals.viewport[0] = float(size)
    f.globals.viewport[1] = float(size)
    ring = ringed([0.0, 4.0, -2.0], 0.1, [0.0, 0.0, 1.0], 0.4)
    ring.ring_params[0] = 100.0
    ring.ring_color[:] = [0.0, 0.0, 0.0, 0.0]
    f.bodies = [body([0.0, 0.0, -5.0], 1.0, [0.8] * 3, False), body([0.0, 4.0, 2.0], 3.8, [1.0] * 3, True), ring]
    direct = float(sample(tracer, f, 4)[:, 0].astype(np.float64).mean())
    tracer.update_options(max_bounces=2)
    mis = float(sample(tracer, f, 4)[:, 0].astype(np.float64).mean())
    assert abs(mis / direct - 1.0) < 0.01, (mis, direct)
    return direct, mis


# ---------------------------------------------------------------------------
# src/ground_tests.rs:1052-1153 — gpu_shadow_queries_match_closest_hits
# (the ring scene; the surface scene needs the local landscape)
# ---------------------------------------------------------------------------
def shadow_ring_scene():
    f = frame()
    ring = body([1.8, 0.0, -5.0], 1.0, [0.0] * 3, False)
    ring.ring_plane[:] = [0.0, 0.8, 0.6, 1.25]
    ring.ring_params[:] = [2.4, 0.7, 0.0, 0.0]
    f.bodies = [
        ring,
        body([0.0, 0.0, -10.0], 0.5, [1.0] * 3, True),
        body([0.0, 0.0, -10.0], 0.5, [1.0] * 3, True),  # equal-distance tie
        body([0.0, 0.0, -20.0], 1.0, [0.5] * 3, False),
    ]
    return f


def shadow_rays(tracer_like_sample_light, f, width: int = 64, height: int = 16):
    """Rays of the shadow probe (src/ground_tests.rs:1079-1093): toward a
    sampled point of light `x % bodies`, or a random direction on rows with
    bit 2 set. `tracer_like_sample_light(f, ray, light, rng) -> (dir, rng)`."""
    n_bodies = len(f.bodies)
    offsets, dirs, lights = [], [], []
    from oracle.binding import oracle_random  # test infrastructure
    for y in range(height):
        for x in range(width):
            pixel = y * width + x
            rng = (pixel * 747796405 + 2891336453) & 0xFFFFFFFF
            light = x % n_bodies
            d, rng = tracer_like_sample_light(f, light, rng)
            if y & 4:
                a, rng = oracle_random(rng)
                b, rng = oracle_random(rng)
                c, rng = oracle_random(rng)
                v = np.array([a, b, c], np.float32) - np.float32(0.5)
                d = v * (np.float32(1.0) / np.sqrt(np.float32(v @ v)))
            offsets.append([0.0, 0.0, 0.0])
            dirs.append(d)
            lights.append(light)
    return rays_array(offsets, dirs, abi.MISS), np.array(lights, np.uint32)


# ---------------------------------------------------------------------------
# Local landscape (src/ground_tests.rs)
# ---------------------------------------------------------------------------
def local_frame(radius_m: float):
    """`local_frame` (src/ground_tests.rs:191-206): a camera 2 m above a host
    sphere, looking 26.6 degrees down, a star up and to the south."""
    f32 = np.float32
    f = frame()
    metre = f32(1.0) / f32(149_597_870_700.0)
    up = np.array([0.0, np.sqrt(f32(0.8)), np.sqrt(f32(0.2))], dtype=np.float32)
    north = np.array([0.0, -up[2], up[1]], dtype=np.float32)
    f.globals.ground_east[:] = [1.0, 0.0, 0.0, 2.0]
    f.globals.ground_up[:] = [float(up[0]), float(up[1]), float(up[2]), float(radius_m)]
    f.globals.ground_north[:] = [float(north[0]), float(north[1]), float(north[2]), 1.0]
    center = -up * ((f32(radius_m) + f32(2.0)) * metre)
    sun = (up * f32(8.0) - north * f32(4.0)) * metre
    f.bodies = [body(center, f32(radius_m) * metre, [0.3] * 3, False), body(sun, f32(0.5) * metre, [100.0] * 3, True)]
    return f


def local_ground_shadows(make) -> dict:
    """`gpu_local_ground_shadows` (src/ground_tests.rs:229-269)."""
    from stargaze_b200.terrain import primitive

    tracer = make((1, 1), test_options(samples_per_frame=64, max_bounces=1))
    out = {}
    for radius in (6_371_000.0, 1_500_000.0):
        scene = local_frame(radius)
        full = float(sample(tracer, scene, 8)[0][0])
        assert full > 0.01 and np.isfinite(full), ("ground unlit", radius, full)
        # A nearby box blocks the star without blocking the camera's ground ray.
        scene.ground.append(primitive([0.0, 4.0, -4.0], 0.0, [0.8, 0.8, 0.8], 0.0, [0, 0, 0], 0.0))
        scene.globals.ground_counts[0] = 1
        box = float(sample(tracer, scene, 8)[0][0])
        assert box < full * 0.001, ("box shadow", radius, box, full)
        scene.ground[0].center[3] = 1.0
        ellipsoid = float(sample(tracer, scene, 8)[0][0])
        assert ellipsoid < full * 0.001, ("ellipsoid shadow", radius, ellipsoid, full)
        # A blocker two centimetres above the surface must also shadow it.
        scene.ground[0].center[:] = [0.0, 0.02, -4.0, 0.0]
        scene.ground[0].extent[:] = [0.2, 0.004, 0.005, 0.0]
        small = float(sample(tracer, scene, 8)[0][0])
        assert small < full * 0.01, ("centimetre shadow", radius, small, full)
        # Rotated boxes take part in visibility too.
        scene.ground[0].center[:] = [0.0, 4.0, -4.0, 0.0]
        scene.ground[0].extent[:] = [0.8, 0.8, 0.8, 0.4]
        rotated = float(sample(tracer, scene, 8)[0][0])
        assert rotated < full * 0.001, ("rotated box shadow", radius, rotated, full)
        out[radius] = dict(full=full, box=box, ellipsoid=ellipsoid, small=small, rotated=rotated)
    return out


# Rays of heightfield_oracle (src/ground_tests.rs:749-760), surface frame at
# terrain scale 1; origins are multiplied by the terrain scale.
HEIGHTFIELD_RAYS = [
    ([0.0, 300.0, 0.0], [0.0, -1.0, 0.0]),
    ([0.0, 2.0, 0.0], [0.0, 0.03, 1.0]),
    ([0.0, 2.0, 0.0], [1.0, 0.08, 0.25]),
    ([0.0, 2.0, 0.0], [-1.0, 0.1, -0.4]),
    ([0.0, 2.0, 0.0], [0.0, 1.0, 0.0]),
    ([1_000.0, 2_000.0, -3_000.0], [0.0, -1.0, 0.0]),
    ([-4_000.0, 1_500.0, 2_000.0], [1.0, -0.2, 0.1]),
    ([16_000.0, 100.0, 0.0], [0.0, -1.0, 0.0]),
    ([16_100.0, 100.0, 0.0], [0.0, -1.0, 0.0]),
    ([0.0, 0.1, 0.0], [0.5, -0.01, -1.0]),
]


def terrain_frame(radius_m: float):
    """A frame whose landscape uses the uploaded terrain (forest theme)."""
    f = local_frame(radius_m)
    f.globals.ground_counts[1] = 1
    return f


def exhaustive_terrain_hit(heights: np.ndarray, cells: int, radius_m: float, o, d) -> float:
    """Independent f64 exhaustive intersection of the triangulated
    heightfield, as src/ground_tests.rs:738-747 and :817-848 do: no quadtree,
    bounds or traversal."""
    from stargaze_b200.terrain import coordinates, terrain_scale

    scale = terrain_scale(radius_m)
    c = coordinates(cells, 1.0).astype(np.float64) * scale
    width = cells + 1
    x, z = np.meshgrid(c, c)
    r = float(np.float32(radius_m))
    curvature = -(x * x + z * z) / (r + np.sqrt(r * r - x * x - z * z))
    y = np.asarray(heights, np.float64).reshape(width, width) * scale + curvature
    V = np.stack([x, y, z], axis=-1)
    a, b, cc, e = V[:-1, :-1], V[:-1, 1:], V[1:, :-1], V[1:, 1:]
    o = np.asarray(o, np.float64)
    d = np.asarray(d, np.float64)

    def tri(A, B, C):
        ab, ac = B - A, C - A
        p = np.cross(d, ac)
        det = np.sum(ab * p, axis=-1)
        with np.errstate(divide="ignore", invalid="ignore"):
            rel = o - A
            u = np.sum(rel * p, axis=-1) / det
            q = np.cross(rel, ab)
            v = np.sum(d * q, axis=-1) / det
            t = np.sum(ac * q, axis=-1) / det
        ok = (np.abs(det) >= 1e-15) & (u >= -1e-9) & (v >= -1e-9) & (u + v <= 1 + 1e-9) & (t > 0.001)
        return np.where(ok, t, np.inf)

    return float(min(tri(a, cc, b).min(), tri(e, b, cc).min()))


def heightfield_oracle(make, heights: np.ndarray, data: np.ndarray, cells: int, rays=None) -> list:
    """`heightfield_oracle` (src/ground_tests.rs:691-903) on a seeded fBm grid:
    quadtree hits within 0.005 m + 1e-5 t of the exhaustive f64 scan, misses
    where it misses, unit normals pointing up."""
    from stargaze_b200.terrain import terrain_scale

    rays = HEIGHTFIELD_RAYS if rays is None else rays
    results = []
    for radius in (6_371_000.0, 5_000.0):
        tracer = make((1, 1), test_options())
        tracer.upload_terrain(data, cells)
        f = terrain_frame(radius)
        scale = np.float32(terrain_scale(radius))
        origins = np.array([np.float32(o) * scale for o, _ in [(np.array(o, np.float32), d) for o, d in rays]])
        dirs = []
        for _, d in rays:
            d = np.array(d, np.float32)
            dirs.append(d * (np.float32(1.0) / np.sqrt(np.float32(d @ d))))
        dirs = np.array(dirs, np.float32)
        out = tracer.terrain_probe(f, origins, dirs)
        for k in range(len(rays)):
            expected = exhaustive_terrain_hit(heights, cells, radius, origins[k], dirs[k])
            actual = float(out[k][3])
            if np.isinf(expected):
                assert actual > 1e29, (radius, k, out[k])
            else:
                assert abs(actual - expected) < 0.005 + expected * 1e-5, (radius, k, actual, expected)
                n = out[k][:3]
                assert np.all(np.isfinite(n)) and abs(np.linalg.norm(n) - 1.0) < 1e-4 and n[1] > 0.0, (radius, k, n)
            results.append((radius, k, actual, expected))
    return results


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:842-994 — gpu_atmosphere
# ---------------------------------------------------------------------------
AU_KM = 149_597_870.7


def earthlike() -> dict:
    """`Atmosphere::earthlike` (src/sim.rs:295-306), coefficients per AU."""
    au_m = AU_KM * 1000.0
    return dict(scale_height=8500.0 / au_m, thickness=80000.0 / au_m,
                rayleigh=[5.8e-6 * au_m, 13.5e-6 * au_m, 33.1e-6 * au_m], mie=21.0e-6 * au_m, mie_g=0.76)


def dense() -> dict:
    """`Atmosphere::dense` (src/sim.rs:287-292): three times the scattering."""
    a = earthlike()
    a["rayleigh"] = [b * 3.0 for b in a["rayleigh"]]
    a["mie"] *= 3.0
    return a


def set_air(f, a: dict, center, radius: float, host: float = 1.0) -> None:
    f.globals.atmo_center[:] = [center[0], center[1], center[2], radius]
    f.globals.atmo_rayleigh[:] = [*a["rayleigh"], a["mie"]]
    f.globals.atmo_params[:] = [a["mie_g"], a["scale_height"], a["thickness"], host]


def catalogue_star(bright: float = 1.0) -> dict:
    return dict(dir=[0.0, 0.0, -1.0], color=[1.0, 1.0, 1.0], bright=bright, angular_radius=0.01)


def atmosphere(make) -> dict:
    from stargaze_b200 import sky

    opts = test_options(samples_per_frame=64, max_bounces=1, exposure=1.0)
    background = catalogue_star()
    tracer = make((1, 1), opts)
    tracer.upload_catalogue(*sky.ray_catalogue([background]))
    f = frame()
    a = earthlike()
    radius = np.float32(6371.0 / AU_KM)
    # The camera looks straight up, two metres above the host surface.
    center = [0.0, 0.0, float(np.float32(radius + np.float32(0.002 / AU_KM)))]
    f.bodies = [body(center, float(radius), [0.0] * 3, False)]
    set_air(f, a, center, float(radius))
    attenuated = sample(tracer, f, 1)[0]
    star = sky.radiance(background)
    # Eight midpoint cells integrate an exponential profile to exactly
    # x / (2 sinh(x / 2)) times the continuous column, x one cell's
    # thickness in scale heights.
    h, top = a["scale_height"], a["thickness"]
    column = h * (math.exp(-0.002 / AU_KM / h) - math.exp(-top / h))
    x = (top - 0.002 / AU_KM) / (8.0 * h)
    midpoint = column * x / (2.0 * math.sinh(x * 0.5))
    for c in range(3):
        expected = float(np.float32(math.exp(-(a["rayleigh"][c] + a["mie"]) * midpoint))) * star[c]
        assert abs(attenuated[c] - expected) < 0.001 * expected, (c, attenuated[c], expected)
    f.globals.atmo_params[3] = 0.0
    unattenuated = sample(tracer, f, 1)[0]
    for c in range(3):
        assert abs(unattenuated[c] - star[c]) <= 1e-5 * star[c], (unattenuated, star)
    assert unattenuated[3] == 0.0
    f.globals.atmo_params[3] = 1.0

    # No catalogue: any light in this zenith ray comes from scattering.
    tracer = make((1, 1), opts)
    f.bodies.append(body([1.0, 0.0, -1.0], 0.005, [100_000.0] * 3, True))
    day = sample(tracer, f, 4)[0]
    assert np.all(np.isfinite(day[:3])) and np.all(day[:3] > 0.01), day
    assert day[2] > day[0], day
    f.bodies.append(body([0.5, 0.0, -0.5], 0.05, [0.0] * 3, False))
    eclipsed = sample(tracer, f, 4)[0]
    assert np.array_equal(eclipsed, np.zeros(4, np.float32)), eclipsed
    f.bodies.pop()
    f.bodies[1].center[:] = [1.0, 0.0, 0.03]
    twilight = sample(tracer, f, 4)[0]
    assert twilight[0] > 0.0001, twilight
    f.bodies[1].center[:] = [0.0, 0.0, 1.0]
    assert np.array_equal(sample(tracer, f, 1)[0], np.zeros(4, np.float32))

    # Dense haze hides the catalogue by day, keeps it by night and while an
    # eclipse shadows the air.
    d = dense()
    f.globals.atmo_rayleigh[:] = [*d["rayleigh"], d["mie"]]
    bright = catalogue_star(1.62)
    with_stars = make((1, 1), opts)
    with_stars.upload_catalogue(*sky.ray_catalogue([bright]))
    night = sample(with_stars, f, 4)[0]
    star = sky.radiance(bright)
    assert night[0] > 0.3 * star[0], night
    f.bodies[1] = body([1.0, 0.0, -1.0], 0.005, [44_444.0] * 3, True)
    day_sky = sample(tracer, f, 4)[0]
    day_stars = sample(with_stars, f, 4)[0]
    for c in range(3):
        assert abs(day_stars[c] - day_sky[c]) < 0.03 * day_sky[c], (day_stars, day_sky)
    f.bodies.append(body([0.5, 0.0, -0.5], 0.05, [0.0] * 3, False))
    eclipse = sample(with_stars, f, 4)[0]
    for c in range(3):
        assert abs(eclipse[c] - night[c]) < 0.01 * night[c] + 1e-9, (eclipse, night)
    return dict(attenuated=attenuated, day=day, twilight=twilight, night=night, day_sky=day_sky,
                day_stars=day_stars, eclipse=eclipse)


# ---------------------------------------------------------------------------
# src/pathtracer_tests.rs:996-1104 — gpu_reflected_atmosphere
# ---------------------------------------------------------------------------
def reflected_atmosphere(make) -> dict:
    """The glow is the difference of two renders. The reference takes them
    from one tracer (independent noise sequences); the daylight case then
    compares the day sky's noise, about 2e-4 of it at 2048 samples (the Mie
    lobe varies by +-2.5 % across the sun's disc), with 2 % of the glow. Here
    both renders use the same sequence (common random numbers): planetshine
    draws from its own stream, so the difference is the glow alone."""
    opts = test_options(samples_per_frame=64, max_bounces=1)
    f = frame()
    a = earthlike()
    radius = np.float32(6371.0 / AU_KM)
    center = [0.0, 0.0, float(np.float32(radius + np.float32(0.002 / AU_KM)))]
    set_air(f, a, center, float(radius))
    # A large moon just outside the zenith ray; the sun is below the host's
    # horizon but lights the moon without a lunar eclipse.
    f.bodies = [body(center, float(radius), [0.0] * 3, False),
                body([0.0004, 0.0, -0.002], 0.00015, [0.8] * 3, False),
                body([0.3, 0.0, 1.0], 0.005, [100_000.0] * 3, True)]

    def glow():
        color = list(f.bodies[1].color)
        f.bodies[1].color[:] = [0.0] * 3
        background = sample(make((1, 1), opts), f, 32)[0]
        f.bodies[1].color[:] = color
        lit = sample(make((1, 1), opts), f, 32)[0]
        return np.array([lit[c] - background[c] for c in range(3)], np.float64)

    full = glow()
    assert np.all(np.isfinite(full)) and np.all(full > 1e-4), full
    f.bodies[1].color[:] = [0.4, 0.2, 0.1]
    tinted = glow()
    for c in range(3):
        expected = full[c] * [0.5, 0.25, 0.125][c]
        assert abs(tinted[c] - expected) < expected * 0.02, (tinted, full)
    f.bodies[1].color[:] = [0.8] * 3
    f.bodies[1].radius *= 0.5
    small = glow()
    assert full[0] * 0.15 < small[0] < full[0] * 0.35, (small, full)
    f.bodies[1].radius *= 2.0
    f.bodies[2].center[:] = [1.0, 0.0, 0.0]
    quarter = glow()
    f.bodies[2].center[:] = [-0.3, 0.0, -1.0]
    new = glow()
    assert full[0] * 0.1 < quarter[0] < full[0] * 0.6, (quarter, full)
    assert abs(new[0]) < full[0] * 0.02, (new, full)
    f.bodies[2].center[:] = [0.3, 0.0, 1.0]
    # Starlight blocked on its way to the moon.
    f.bodies.append(body([0.1502, 0.0, 0.499], 0.01, [0.0] * 3, False))
    eclipsed = glow()
    assert np.all(np.abs(eclipsed) < 1e-6), eclipsed
    f.bodies.pop()
    # Moonlight blocked on its way to the air.
    f.bodies.append(body([0.0002, 0.0, -0.001], 0.00012, [0.0] * 3, False))
    hidden = glow()
    assert np.all(np.abs(hidden) < 1e-6), hidden
    f.bodies.pop()
    f.globals.atmo_params[3] = 0.0
    airless = glow()
    assert np.all(np.abs(airless) < 1e-6), airless
    return dict(full=full, tinted=tinted, small=small, quarter=quarter, new=new)


# ---------------------------------------------------------------------------
# The guided ground sampler (src/guided_ground.rs:14-79)
# ---------------------------------------------------------------------------
def moonlit_ground_frame(size: int = 4):
    """`local_frame` at night under earthlike air: the star set 17 degrees
    below the horizon, a large sunlit moon (0.1 rad across, albedo 0.5) high
    in the south. The ground sees the moon only through continuations (the
    moon is not a light), the case the guided sampler aims at."""
    f = local_frame(6_371_000.0)
    f.globals.viewport[:] = [float(size), float(size), 1.0, 1.0]
    f.globals.cam_forward[3] = 0.05
    host = f.bodies[0]
    set_air(f, earthlike(), list(host.center), host.radius, host=1.0)
    up = np.array(f.globals.ground_up[:3], np.float64)
    north = np.array(f.globals.ground_north[:3], np.float64)
    sun_dir = -0.3 * up + north
    sun_dir /= np.linalg.norm(sun_dir)
    f.bodies[1] = body(list(sun_dir * 1.0), 0.00465, [40_000.0] * 3, True)
    moon_dir = 0.8 * up - 0.6 * north
    moon_dir /= np.linalg.norm(moon_dir)
    d = 3.0e-4
    f.bodies.append(body(list(moon_dir * d), d * 0.05, [0.5] * 3, False))
    return f


def guided_ground_is_unbiased(make, batches: int = 24) -> dict:
    """Plain and guided estimates of the moonlit ground agree; the guided
    one has the lower variance. Batch means give the standard errors."""
    f = moonlit_ground_frame()
    out = {}
    for guided in (False, True):
        means = []
        for k in range(batches):
            t = make((4, 4), test_options(samples_per_frame=64, max_bounces=3, noise_seed=1000 * k + 7))
            t.set_guided_ground(guided)
            means.append(float(sample(t, f, 1)[:, :3].mean()))
        m = np.array(means)
        out[guided] = (m.mean(), m.std(ddof=1) / np.sqrt(len(m)))
    (mp, sp), (mg, sg) = out[False], out[True]
    assert mg > 0.0 and mp > 0.0, out
    assert abs(mg - mp) < 4.0 * np.hypot(sp, sg), out
    assert sg < sp, out
    return dict(plain=out[False], guided=out[True])


# ---------------------------------------------------------------------------
# src/planetshine_tests.rs:53-104 — gpu_textured_planets_light_night_air
# ---------------------------------------------------------------------------
STYLES = ["gas_giant", "cratered", "rocky", "icy", "volcanic", "terran"]


def default_surface(style: str, albedo) -> dict:
    """`config::default_surface` (src/config.rs:191-290): a style's
    defaults for a body of `albedo` (secondary colour, bands, turbulence,
    storms, craters, ice caps, ocean, clouds)."""
    a = np.asarray(albedo, np.float32)
    peak = np.float32(max(1.0e-6, float(a.max())))

    def deeper(scale, power):
        return [float(np.float32(scale) * c * np.float32(np.power(np.float32(c / peak), np.float32(power)))) for c in a]

    secondary = {
        "gas_giant": lambda: deeper(0.8, 1.6), "cratered": lambda: deeper(0.55, 0.6),
        "rocky": lambda: deeper(0.6, 1.0), "icy": lambda: [a[0] * 0.75, a[1] * 0.5, a[2] * 0.35],
        "volcanic": lambda: [a[0] * 0.85, a[1] * 0.45, a[2] * 0.2], "terran": lambda: [0.03, 0.09, 0.2],
    }[style]()
    craters, ice_caps = {"gas_giant": (0.0, 0.0), "cratered": (0.8, 0.0), "rocky": (0.5, 0.06), "icy": (0.15, 0.0),
                         "volcanic": (0.5, 0.0), "terran": (0.0, 0.1)}[style]
    return dict(code=float(STYLES.index(style) + 1), secondary=[float(c) for c in secondary], bands=7.0,
                turbulence=0.5, storms=1, craters=craters, ice_caps=ice_caps, ocean=0.65, clouds=0.4)


def texture(sphere, style: str) -> None:
    """`texture` (src/planetshine_tests.rs:30-51): a style's defaults on a
    body, pattern seed 17, body axes along x and y."""
    s = default_surface(style, list(sphere.color))
    gas = style == "gas_giant"
    sphere.axis_x[:] = [1.0, 0.0, 0.0, s["code"]]
    sphere.axis_y[:] = [0.0, 1.0, 0.0, 17.0]
    sphere.surface_color[:] = [*s["secondary"], s["turbulence"] if gas else s["craters"]]
    sphere.surface_params[:] = ([s["bands"], float(s["storms"]), 0.0, 0.0] if gas
                                else [s["ice_caps"], s["ocean"], s["clouds"], 0.0])


def moonlit_scene():
    """`moonlit_scene` (src/planetshine_tests.rs:4-28)."""
    f = frame()
    radius = np.float32(6371.0 / AU_KM)
    center = [0.0, 0.0, float(np.float32(radius + np.float32(0.002 / AU_KM)))]
    set_air(f, earthlike(), center, float(radius))
    f.bodies = [body(center, float(radius), [0.0] * 3, False),
                body([0.0004, 0.0, -0.002], 0.00015, [0.8, 0.6, 0.4], False),
                body([0.3, 0.0, 1.0], 0.005, [100_000.0] * 3, True)]
    return f


def textured_planets_light_night_air(make, styles=STYLES) -> dict:
    """Every textured style lights the night air with the right phase and no
    glow from its unlit face. The glow is lit minus an untextured black moon;
    both renders use the same sequence (common random numbers), as in
    `reflected_atmosphere`."""
    opts = test_options(samples_per_frame=32, max_bounces=1)
    out = {}
    for style in styles:
        scene = moonlit_scene()
        texture(scene.bodies[1], style)

        def glow(scene):
            lit = sample(make((1, 1), opts), scene, 32)[0]
            black = moonlit_scene()
            black.bodies[1] = type(scene.bodies[1]).from_buffer_copy(scene.bodies[1])
            black.bodies[1].color[:] = [0.0] * 3
            black.bodies[1].axis_x[3] = 0.0
            black.bodies[2] = type(scene.bodies[2]).from_buffer_copy(scene.bodies[2])
            background = sample(make((1, 1), opts), black, 32)[0]
            return np.array([lit[c] - background[c] for c in range(3)], np.float64)

        full = glow(scene)
        scene.bodies[2].center[:] = [1.0, 0.0, 0.0]
        quarter = glow(scene)
        scene.bodies[2].center[:] = [-0.3, 0.0, -1.0]
        new = glow(scene)
        assert np.all(np.isfinite(full)) and np.all(full > 1e-4), (style, full)
        assert full[0] * 0.03 < quarter[0] < full[0] * 0.8, (style, quarter, full)
        assert np.all(np.abs(new) < full * 0.03), (style, new, full)
        out[style] = dict(full=full, quarter=quarter, new=new)
    return out


def styles_scene(width: int = 96, height: int = 32):
    """Six textured planets in a row (one per style, their defaults, pattern
    seed 17), a star above and behind the camera, tan(half field) 0.17."""
    f = frame()
    f.globals.viewport[:] = [float(width), float(height), 1.0, width / height]
    f.globals.cam_forward[3] = 0.17
    colours = [[0.85, 0.7, 0.5], [0.5, 0.5, 0.48], [0.75, 0.45, 0.3], [0.9, 0.88, 0.85], [0.9, 0.8, 0.35],
               [0.55, 0.5, 0.35]]
    f.bodies = []
    for k, style in enumerate(STYLES):
        b = body([(k - 2.5) * 2.1, 0.0, -12.0], 0.95, colours[k], False)
        texture(b, style)
        # Tilt each body's axes so its pole leans toward the camera.
        b.axis_x[:3] = [1.0, 0.0, 0.0]
        b.axis_y[:3] = [0.0, 0.6, 0.8]
        f.bodies.append(b)
    f.bodies.append(body([4.0, 30.0, 20.0], 1.5, [400.0] * 3, True))
    return f
