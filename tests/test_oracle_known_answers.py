"""The reference's known-answer tests against the CPU oracle (no GPU).

These pin the oracle: every assertion is the reference's own
(src/pathtracer_tests.rs, src/ring_tests.rs, src/ground_tests.rs).
"""
import numpy as np
import pytest

import known_answers as ka
from oracle.binding import OracleTracer, oracle_hash, oracle_random
from stargaze_b200 import abi


def make(dimensions, options):
    return OracleTracer(dimensions, options)


def test_transport():
    r = ka.transport(make)
    assert r["umbra"] < r["penumbra"] < r["annular"] < r["full"]


def test_distant_surface():
    counts = ka.distant_surface(make, size=128)
    assert all(v == 0 for v in counts.values())


def test_noise_sequence():
    ka.noise_sequence(make)


def test_quality_limits_rest_resume():
    ka.quality_limits(make)


def test_rings_geometry():
    ka.rings_geometry(make)


def test_rings_transport():
    ka.rings_transport(make)


def test_rings_conserve_energy():
    energies = ka.rings_conserve_energy(make)
    assert len(energies) == 36


def test_rings_null_crossings_preserve_mis():
    ka.rings_null_crossings_preserve_mis(make, size=32)


@pytest.mark.parametrize("stars", range(6))
def test_shadow_queries_match_closest_hits(stars):
    tracer = OracleTracer((64, 16), ka.test_options())
    f = ka.shadow_ring_scene()
    for i, b in enumerate(f.bodies):
        b.emissive = 1.0 if i < stars else 0.0
    s = f.settings(64, 16, 0, 0, 8, 0)

    def sample_light(frame_, light, rng):
        import ctypes as C
        from oracle.binding import load
        lib = load()
        st = C.c_uint32(rng)
        d = np.zeros(3, np.float32)
        pdf = C.c_float()
        ray = abi.Ray()
        ray.anchor = abi.MISS
        bodies = frame_.bodies_array()
        lib.oracle_sample_light(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(ray), light, C.byref(st),
                                C.c_void_p(d.ctypes.data), C.byref(pdf))
        return d, st.value

    rays, lights = ka.shadow_rays(sample_light, f)
    vis = tracer.light_visibility(f, rays, lights)
    ref = tracer.reference_visibility(f, rays, lights)
    assert np.array_equal(vis, ref)
    # Compact light list == full scan (src/ground_tests.rs:1094-1103).
    compact = 0
    count = s.lights[3] if s.lights[3] <= 3 else s.counts[0]
    for slot in range(count):
        i = s.lights[slot] if s.lights[3] <= 3 else slot
        if f.bodies[i].emissive >= 0.5:
            compact = (compact * 31 + i + 1) & 0xFFFFFFFF
    reference = 0
    for i, b in enumerate(f.bodies):
        if b.emissive >= 0.5:
            reference = (reference * 31 + i + 1) & 0xFFFFFFFF
    assert compact == reference


def _hash_np(x: int) -> int:
    """Independent restatement of hash() (pathtrace.wgsl:87-92)."""
    m = 0xFFFFFFFF
    x &= m
    x = ((x ^ (x >> 16)) * 0x7FEB352D) & m
    x = ((x ^ (x >> 15)) * 0x846CA68B) & m
    return x ^ (x >> 16)


def _random_np(state: int):
    m = 0xFFFFFFFF
    state = (state * 747796405 + 2891336453) & m
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & m
    return float(np.float32(((word >> 22) ^ word) >> 8) * np.float32(1.0 / 16777216.0)), state


@pytest.mark.parametrize("seed", [0, 1, 0x9E3779B9, 0xFFFFFFFF, 123456789])
def test_rng_matches_wgsl(seed):
    assert oracle_hash(seed) == _hash_np(seed)
    state = _hash_np(seed)
    ostate = state
    for _ in range(16):
        a, state = _random_np(state)
        b, ostate = oracle_random(ostate)
        assert a == b and state == ostate
        assert 0.0 <= a < 1.0


def test_atmosphere():
    r = ka.atmosphere(make)
    assert r["day"][2] > r["day"][0]


def test_reflected_atmosphere():
    r = ka.reflected_atmosphere(make)
    assert r["small"][0] < r["full"][0]


def test_air_frames_are_not_differentiated():
    f = ka.frame()
    ka.set_air(f, ka.earthlike(), [0.0, 0.0, 1e-4], 4e-5)
    tracer = make((2, 2), ka.test_options())
    with pytest.raises(Exception):
        tracer.tangent(f, 0, 1)


def test_guided_ground_is_unbiased():
    r = ka.guided_ground_is_unbiased(make)
    assert r["guided"][1] < r["plain"][1]


def test_textured_planets_light_night_air():
    r = ka.textured_planets_light_night_air(make)
    assert set(r) == set(ka.STYLES)


def test_guided_ground_is_inert_without_air_or_reflectors():
    """The guided sampler only acts at depth-0 local surfaces under air with
    a reflecting body (src/guided_ground.rs:38-48): elsewhere it draws no
    random numbers, so the images are identical."""
    base = ka.moonlit_ground_frame()
    cases = []
    airless = base.copy()
    airless.globals.atmo_params[3] = 0.0
    cases.append(airless)
    no_reflector = base.copy()
    no_reflector.bodies[2].color[:] = [0.0, 0.0, 0.0]
    cases.append(no_reflector)
    for f in cases:
        imgs = []
        for guided in (False, True):
            t = make((4, 4), ka.test_options(samples_per_frame=64, max_bounces=3))
            t.set_guided_ground(guided)
            imgs.append(ka.sample(t, f, 1))
        assert np.array_equal(imgs[0], imgs[1])
    # With air and a lit moon it does change the estimate's samples.
    imgs = []
    for guided in (False, True):
        t = make((4, 4), ka.test_options(samples_per_frame=64, max_bounces=3))
        t.set_guided_ground(guided)
        imgs.append(ka.sample(t, base, 1))
    assert not np.array_equal(imgs[0], imgs[1])


def test_surface_sky_cache_holds_air_light_over_terrain_only():
    """cache_surface_sky (terrain.wgsl:286-302): air light in 16 x 8
    directions of the local sky when both the host air and the terrain are
    on, zero otherwise; a daylit sky is bluer toward the zenith than the
    horizon is reddened."""
    cells = 64
    from stargaze_b200 import terrain as T

    heights = T.fbm_heights(cells, seed=2)
    data = T.pack_terrain(heights, cells)
    f = ka.terrain_frame(6_371_000.0)
    host = f.bodies[0]
    ka.set_air(f, ka.earthlike(), list(host.center), host.radius, host=1.0)
    # A sun high in the south (the local frame's up and north).
    up = np.array(f.globals.ground_up[:3], np.float64)
    north = np.array(f.globals.ground_north[:3], np.float64)
    sun = 0.8 * up - 0.6 * north
    f.bodies[1] = ka.body(list(sun / np.linalg.norm(sun)), 0.00465, [40_000.0] * 3, True)
    t = make((1, 1), ka.test_options())
    t.upload_terrain(data, cells)
    lit = t.sky_cache(f)
    assert np.isfinite(lit).all() and (lit[..., :3] > 0.0).all()
    assert (lit[..., 3] == 0.0).all()
    zenith = lit[7].mean(axis=0)
    assert zenith[2] > zenith[0], zenith
    no_terrain = f.copy()
    no_terrain.globals.ground_counts[1] = 0
    assert (t.sky_cache(no_terrain) == 0.0).all()
    no_air = f.copy()
    no_air.globals.atmo_params[3] = 0.0
    assert (t.sky_cache(no_air) == 0.0).all()
