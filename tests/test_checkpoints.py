"""Vertex checkpoints (sg_set_checkpoints) against path replay.

With checkpoints the forward stores each path's state whenever a scatter
brings its depth to a multiple of `every`, and each sample's radiance; the
backward replays every sample up to its first checkpoint and each later
segment from its record. The paths, their decisions and the derivative
terms are the replay's, so on the same tape the gradients must equal the
replay's to the tolerance the staged and per-pixel adjoints are held to
(test_wave_adjoint.py: accumulation order, and the few paths whose decisions
differ by an ulp between kernel compilations). Samples whose ring-indirect
cap binds, or whose records do not fit the budget, fall back to replay.
"""
import numpy as np
import pytest

from stargaze_b200 import workloads as W
from stargaze_b200.pathtracer import PathTracer
from test_wave_adjoint import assert_same_gradient

pytestmark = pytest.mark.gpu


def forward_backward(wl, spp, seed, land=None, every=0, record_bytes=0):
    t = PathTracer((wl.width, wl.height), W.render_options(wl, 4, noise_seed=seed))
    W.upload_workload(t, wl)
    if land is not None and land.albedo_map is not None:
        t.upload_albedo_map(land.albedo_map, land.map_extent)
    t.set_integrator("wavefront")
    if every:
        t.set_checkpoints(every, spp, record_bytes)
    frame = wl.frame.copy()
    while t.samples() < spp:
        t.encode(frame)
    image = t.read_pixels()
    stats = t.checkpoint_stats()
    tape = t.tape()
    dl = np.random.default_rng(seed).uniform(-1.0, 1.0, (wl.width * wl.height, 4)).astype(np.float32)
    grads = t.backward(frame, tape, dl)
    t.close()
    return image, grads, stats


def terrain_case():
    wl, land = W.terrain_1080p(96, 64, 8, cells=256, rocks=60, foliage=60)
    land.albedo_map = np.random.default_rng(2).uniform(0.05, 0.6, (64, 64)).astype(np.float32)
    land.map_extent = 2000.0
    return wl, land


@pytest.mark.parametrize("every", [1, 2])
def test_checkpointed_adjoint_equals_replay_on_the_terrain_scene(every):
    wl, land = terrain_case()
    img_r, replay, none = forward_backward(wl, 8, 21, land)
    img_c, ckpt, stats = forward_backward(wl, 8, 21, land, every=every)
    assert none["records"] == 0 and stats["records"] > 0 and stats["dropped"] == 0
    assert stats["device_bytes"] >= stats["records"] * 128
    # The checkpointing forward renders the same image.
    np.testing.assert_allclose(img_c, img_r, rtol=1e-5, atol=1e-7)
    assert_same_gradient(ckpt.albedo_map, replay.albedo_map, "albedo_map")
    assert_same_gradient(ckpt.body_color, replay.body_color, "body_color")


@pytest.mark.parametrize("every", [2, 64])
def test_checkpointed_adjoint_equals_replay_on_the_ring_scene(every):
    """Ring scatters, null crossings and the ring-indirect cap (its binding
    samples replay from the seed). every = 64, beyond the bounce limit,
    stores the radiance alone: whole paths replay once with known weights."""
    wl = W.rings_1080p(96, 64, 8)
    _, replay, _ = forward_backward(wl, 8, 22)
    _, ckpt, stats = forward_backward(wl, 8, 22, every=every)
    assert (stats["records"] > 0) == (every < wl.max_bounces)
    assert stats["device_bytes"] >= 96 * 64 * 8 * 16
    assert_same_gradient(ckpt.ring_tau[0, :512], replay.ring_tau[0, :512], "ring_tau")
    assert_same_gradient(ckpt.ring_albedo, replay.ring_albedo, "ring_albedo")
    assert_same_gradient(ckpt.body_color, replay.body_color, "body_color")


def test_records_beyond_the_budget_fall_back_to_replay():
    wl, land = terrain_case()
    _, replay, _ = forward_backward(wl, 8, 23, land)
    _, ckpt, stats = forward_backward(wl, 8, 23, land, every=1, record_bytes=8 * 128)
    assert stats["records"] == 8 and stats["dropped"] > 0
    assert_same_gradient(ckpt.albedo_map, replay.albedo_map, "albedo_map")
