"""The reference's known-answer tests against the CUDA library (B200)."""
import ctypes as C

import numpy as np
import pytest

import known_answers as ka
from stargaze_b200 import PathTracer, abi
from stargaze_b200._lib import StargazeError

pytestmark = pytest.mark.gpu


def make(dimensions, options):
    return PathTracer(dimensions, options)


def test_transport():
    r = ka.transport(make)
    assert r["umbra"] < r["penumbra"] < r["annular"] < r["full"]


def test_distant_surface():
    counts = ka.distant_surface(make, size=256)
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
    assert len(ka.rings_conserve_energy(make)) == 36


def test_rings_null_crossings_preserve_mis():
    ka.rings_null_crossings_preserve_mis(make, size=64)


@pytest.mark.parametrize("stars", range(6))
def test_shadow_queries_match_closest_hits(stars):
    """Any-hit visibility == closest-hit reference, bit-equal
    (src/ground_tests.rs:1052-1153, ring scene)."""
    from oracle.binding import load as load_oracle

    tracer = PathTracer((64, 16), ka.test_options())
    f = ka.shadow_ring_scene()
    for i, b in enumerate(f.bodies):
        b.emissive = 1.0 if i < stars else 0.0
    s = f.settings(64, 16, 0, 0, 8, 0)
    lib = load_oracle()

    def sample_light(frame_, light, rng):
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
    hits = tracer.closest_hit(f, rays)
    ref = np.zeros_like(vis)
    rings = [tracer.ring_probe(f, rays, i) for i in range(len(f.bodies))]
    for k in range(len(rays)):
        if hits["index"][k] != lights[k]:
            continue
        t = np.float32(1.0)
        for i in range(len(f.bodies)):
            p = rings[i][k]
            if p[3] != 0.0 and p[0] < hits["distance"][k]:
                t = np.float32(t * p[2])
        ref[k] = t
    assert np.array_equal(vis, ref)


def test_atmosphere():
    r = ka.atmosphere(make)
    assert r["day"][2] > r["day"][0]


@pytest.mark.parametrize("integrator", ["megakernel", "wavefront"])
def test_reflected_atmosphere(integrator):
    def make_with(dimensions, options):
        t = PathTracer(dimensions, options)
        t.set_integrator(integrator)
        return t

    r = ka.reflected_atmosphere(make_with)
    assert r["small"][0] < r["full"][0]


def test_atmosphere_matches_oracle_pixel_for_pixel():
    """The zenith-sky scenario's renders, CUDA against the oracle: the same
    random sequences through the camera air, planetshine and the fresh
    frame's four-stratum light samples."""
    from oracle.binding import OracleTracer

    outs = []
    for cls in (PathTracer, OracleTracer):
        outs.append(ka.atmosphere(lambda d, o, cls=cls: cls(d, o)))
    cuda, cpu = outs
    for key in cpu:
        ref = np.asarray(cpu[key], np.float64)
        got = np.asarray(cuda[key], np.float64)
        assert np.all(np.abs(got - ref) <= 2e-5 * np.abs(ref) + 1e-12), (key, got, ref)


def test_air_frames_are_not_differentiated():
    f = ka.frame()
    ka.set_air(f, ka.earthlike(), [0.0, 0.0, 1e-4], 4e-5)
    t = PathTracer((2, 2), ka.test_options())
    t.encode(f)
    with pytest.raises(StargazeError, match="host air"):
        t.backward(f, t.tape(), np.ones((4, 4), np.float32))


@pytest.mark.parametrize("integrator", ["megakernel", "wavefront"])
def test_guided_ground_is_unbiased(integrator):
    def make_with(dimensions, options):
        t = PathTracer(dimensions, options)
        t.set_integrator(integrator)
        return t

    ka.guided_ground_is_unbiased(make_with)


@pytest.mark.parametrize("guided", [False, True])
@pytest.mark.parametrize("integrator", ["megakernel", "wavefront"])
def test_moonlit_ground_matches_oracle(integrator, guided):
    """The guided ground sampler and the air's extinction of next-event and
    continuations, CUDA against the oracle on the same random sequences."""
    from oracle.binding import OracleTracer

    f = ka.moonlit_ground_frame(size=8)
    imgs = []
    for cls in (PathTracer, OracleTracer):
        t = cls((8, 8), ka.test_options(samples_per_frame=64, max_bounces=3))
        if cls is PathTracer:
            t.set_integrator(integrator)
        t.set_guided_ground(guided)
        imgs.append(ka.sample(t, f, 2))
    img, ref = imgs
    assert np.isfinite(img).all() and ref[:, :3].mean() > 0.0
    err = np.sqrt(((img[:, :3] - ref[:, :3]) ** 2).sum() / (ref[:, :3] ** 2).sum())
    assert err < 2e-3, err
    close = np.abs(img[:, :3] - ref[:, :3]) <= 1e-4 * np.maximum(np.abs(ref[:, :3]), 1e-3 * ref[:, :3].max())
    assert close.all(axis=1).mean() >= 0.99


@pytest.mark.parametrize("integrator", ["megakernel", "wavefront"])
def test_textured_planets_light_night_air(integrator):
    def make_with(dimensions, options):
        t = PathTracer(dimensions, options)
        t.set_integrator(integrator)
        return t

    r = ka.textured_planets_light_night_air(make_with)
    assert set(r) == set(ka.STYLES)


def test_styled_frames_are_not_differentiated():
    f = ka.styles_scene(8, 4)
    t = PathTracer((8, 4), ka.test_options())
    t.encode(f)
    with pytest.raises(StargazeError, match="surface styles"):
        t.backward(f, t.tape(), np.ones((32, 4), np.float32))
