"""The wavefront integrator (PathTracer.set_integrator("wavefront")) runs the
same per-path functions as the per-pixel megakernel, in stage kernels over
queues of paths in device memory, and resolves each pixel's samples in
sample order. The two are compiled into different kernels, so the compiler
may fuse a shading multiply-add in one and not the other: accumulations
agree to a few ulps rather than bit for bit (hit ids, distances and every
random decision are the same code, but an ulp can flip a decision drawn
within an ulp of its threshold). Bar: 99 % of pixels within 2e-6 relative
and relative RMSE below the oracle bar (2e-3); the oracle parity of both
integrators is in test_cuda_parity.py."""
import numpy as np
import pytest

import golden_io as gio

from stargaze_b200 import workloads as W
from stargaze_b200.pathtracer import PathTracer

pytestmark = pytest.mark.gpu


def assert_same_image(wave, mega):
    assert np.isfinite(wave).all()
    assert gio.relative_rmse(wave, mega) < 2e-3
    close = np.abs(wave[:, :3] - mega[:, :3]) <= 2e-6 * np.maximum(np.abs(mega[:, :3]), 1e-6)
    assert close.all(axis=1).mean() >= 0.99
    np.testing.assert_array_equal(wave[:, 3], mega[:, 3])


def render(wl, integrator: str, dispatches: int, spp: int, pool: int = 0, fp64: bool = False, seed: int = 5):
    t = PathTracer((wl.width, wl.height), W.render_options(wl, spp, noise_seed=seed))
    W.upload_workload(t, wl)
    t.set_integrator(integrator, pool)
    t.set_fp64_sites(fp64)
    frame = wl.frame.copy()
    for _ in range(dispatches):
        t.encode(frame)
    image = t.read_pixels()
    stats = t.integrator()
    samples = t.samples()
    t.close()
    return image, stats, samples


def small_terrain(width, height):
    wl, _ = W.terrain_1080p(width, height, 8, cells=256, rocks=60, foliage=60)
    return wl


SCENES = {
    "spheres": lambda w, h: W.spheres_256(w, h),
    "rings": lambda w, h: W.rings_1080p(w, h),
    "terrain": small_terrain,
}


@pytest.mark.parametrize("scene", sorted(SCENES))
def test_wavefront_equals_megakernel(scene):
    """Two dispatches (the second folds into the compensated sum) on an
    image whose sides are not multiples of the 16-pixel tile."""
    wl = SCENES[scene](100, 70)
    mega, _, n_mega = render(wl, "megakernel", 2, 8)
    wave, stats, n_wave = render(wl, "wavefront", 2, 8)
    assert n_mega == n_wave == 16
    assert stats["integrator"] == "wavefront" and stats["iterations"] > 0
    assert np.abs(mega[:, :3]).sum() > 0
    assert_same_image(wave, mega)


@pytest.mark.parametrize("pool", [256, 1000, 5000])
def test_small_pools_refill_without_changing_the_image(pool):
    """Pools far smaller than the dispatch: paths of many samples share the
    pool, the generate stage refills it every iteration."""
    wl = W.rings_1080p(64, 48)
    mega, _, _ = render(wl, "megakernel", 1, 16)
    wave, stats, _ = render(wl, "wavefront", 1, 16, pool=pool)
    assert stats["pool_paths"] == pool
    assert stats["iterations"] >= 64 * 48 * 16 // pool
    assert_same_image(wave, mega)


def test_wavefront_with_fp64_sites():
    wl = small_terrain(64, 40)
    mega, _, _ = render(wl, "megakernel", 1, 8, fp64=True)
    wave, _, _ = render(wl, "wavefront", 1, 8, fp64=True)
    assert_same_image(wave, mega)


def test_wavefront_splits_large_dispatches_into_sample_chunks():
    """3840x2160 at 32 samples per dispatch needs more than the per-sample
    radiance budget (2.25 GiB at 16 B per pixel and sample), so the dispatch
    runs in two chunks whose per-pixel totals carry over in sample order."""
    wl = W.spheres_256(3840, 2160)
    mega, _, _ = render(wl, "megakernel", 1, 32)
    wave, stats, _ = render(wl, "wavefront", 1, 32)
    assert stats["iterations"] > 0
    assert_same_image(wave, mega)


def test_integrator_choice_is_validated():
    from stargaze_b200._lib import StargazeError

    t = PathTracer((16, 16))
    with pytest.raises(StargazeError):
        t.set_integrator("wavefront", 17)
    with pytest.raises(ValueError):
        t.set_integrator("tiled")
    assert t.integrator()["integrator"] == "wavefront"  # the default
    t.close()


def cluster(width=96, height=64, spp=8):
    """40 bodies in telescope space: four stars (more than the three light
    slots, so lights are found by scanning every body), two ringed planets,
    34 diffuse spheres; seeded."""
    from stargaze_b200.scene import body, frame, ringed

    rng = np.random.default_rng(21)
    f = frame()
    f.globals.viewport[:] = [float(width), float(height), 1.0, width / height]
    f.globals.cam_forward[3] = 0.6
    bodies = []
    for k in range(40):
        c = [rng.uniform(-6, 6), rng.uniform(-4, 4), rng.uniform(-22, -7)]
        if k < 4:
            bodies.append(body(c, rng.uniform(0.2, 0.5), rng.uniform(5, 20, 3), True))
        elif k < 6:
            pole = rng.normal(size=3)
            bodies.append(ringed(c, rng.uniform(0.5, 1.0), pole / np.linalg.norm(pole), 0.6))
            bodies[-1].color[:] = list(rng.uniform(0.2, 0.8, 3))
        else:
            bodies.append(body(c, rng.uniform(0.2, 1.0), rng.uniform(0.1, 0.9, 3), False))
    f.bodies = bodies
    return W.Workload("cluster_40", f, width, height, spp, 8, {}, "40 bodies, 4 stars, 2 rings")


def test_wavefront_equals_megakernel_with_many_bodies():
    wl = cluster()
    mega, _, _ = render(wl, "megakernel", 2, 8)
    wave, stats, _ = render(wl, "wavefront", 2, 8)
    assert np.abs(mega[:, :3]).sum() > 0
    assert_same_image(wave, mega)
