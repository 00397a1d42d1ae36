"""The staged adjoint (sg_backward on a context whose integrator is the
wavefront) replays the same samples with the same derivative hooks as the
per-pixel adjoint kernel, through the extend / ring / surface stages with a
per-path adjoint slot. Its gradients must equal the per-pixel kernel's up
to the order of floating-point accumulation (atomics in both) and the few
paths whose forward decisions differ by an ulp between the two integrators'
compilations. The adjoint's unbiasedness (oracle tangent, finite
differences) is tested in test_cuda_adjoint.py with the default, staged
adjoint."""
import numpy as np
import pytest

from stargaze_b200 import workloads as W
from stargaze_b200.pathtracer import PathTracer

pytestmark = pytest.mark.gpu


def both_adjoints(wl, spp, seed, land=None, pool=0):
    t = PathTracer((wl.width, wl.height), W.render_options(wl, spp, noise_seed=seed))
    W.upload_workload(t, wl)
    if land is not None and land.albedo_map is not None:
        t.upload_albedo_map(land.albedo_map, land.map_extent)
    t.set_integrator("wavefront", pool)
    frame = wl.frame.copy()
    while t.samples() < spp:
        t.encode(frame)
    tape = t.tape()
    dl = np.random.default_rng(seed).uniform(-1.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    staged = t.backward(frame, tape, dl)
    t.set_integrator("megakernel")
    per_pixel = t.backward(frame, tape, dl)
    t.close()
    return staged, per_pixel


def assert_same_gradient(a, b, name):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    scale = float(np.abs(b).max())
    assert scale > 0, name
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    assert rel < 2e-3, (name, rel)
    np.testing.assert_allclose(a, b, rtol=1e-2, atol=2e-3 * scale, err_msg=name)


def test_staged_adjoint_equals_per_pixel_adjoint_on_the_ring_scene():
    wl = W.rings_1080p(128, 96, 16)
    staged, ref = both_adjoints(wl, 16, seed=11)
    assert staged.dropped == 0 and ref.dropped == 0
    assert_same_gradient(staged.ring_tau[0, :512], ref.ring_tau[0, :512], "ring_tau")
    assert_same_gradient(staged.ring_albedo, ref.ring_albedo, "ring_albedo")
    assert_same_gradient(staged.body_color, ref.body_color, "body_color")


def test_staged_adjoint_with_a_small_pool():
    """A pool of 2048 paths: slots are taken and given back many times per
    batch, and pass-2 restarts wait in the pool with their slots."""
    wl = W.rings_1080p(64, 48, 8)
    staged, ref = both_adjoints(wl, 8, seed=12, pool=2048)
    assert_same_gradient(staged.ring_tau[0, :512], ref.ring_tau[0, :512], "ring_tau")
    assert_same_gradient(staged.body_color, ref.body_color, "body_color")


def test_staged_adjoint_equals_per_pixel_adjoint_on_the_terrain_scene():
    wl, land = W.terrain_1080p(96, 64, 8, cells=256, rocks=60, foliage=60)
    land.albedo_map = np.random.default_rng(2).uniform(0.05, 0.6, (64, 64)).astype(np.float32)
    land.map_extent = 2000.0
    staged, ref = both_adjoints(wl, 8, seed=13, land=land)
    assert staged.albedo_map is not None
    assert_same_gradient(staged.albedo_map, ref.albedo_map, "albedo_map")
    assert_same_gradient(staged.body_color, ref.body_color, "body_color")


def test_staged_adjoint_with_many_bodies():
    """The 40-body cluster of test_wavefront.py (four stars, two rings)."""
    from test_wavefront import cluster

    wl = cluster(64, 48, 8)
    staged, ref = both_adjoints(wl, 8, seed=14)
    assert_same_gradient(staged.body_color, ref.body_color, "body_color")
    assert_same_gradient(staged.ring_albedo, ref.ring_albedo, "ring_albedo")
