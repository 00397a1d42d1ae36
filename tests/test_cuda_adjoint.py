"""The CUDA path-replay adjoint (sg_get_tape / sg_backward) against the
oracle's forward-mode tangent on the same samples, and against central
differences of the CUDA forward with common random numbers."""
import ctypes as C

import numpy as np
import pytest

from adjoint_cases import (Direction, apply, body_direction, loss_weights, map_direction, ring_albedo_direction,
                           ring_scene, tau_band, terrain_map_scene)
from oracle.binding import OracleTracer
from stargaze_b200 import abi, workloads as W
from stargaze_b200.pathtracer import PathTracer, StargazeError

pytestmark = pytest.mark.gpu


def cuda_tracer(wl, tables, seed, land=None, albedo_map=None):
    t = PathTracer((wl.width, wl.height), W.render_options(wl, wl.spp, noise_seed=seed))
    for k, v in tables.items():
        t.upload_ring_profile(k, v)
    if land is not None:
        t.upload_terrain(land.terrain, land.cells)
        if albedo_map is not None:
            t.upload_albedo_map(albedo_map, land.map_extent)
    return t


def render_and_backward(wl, seed, dl, land=None):
    amap = None if land is None else land.albedo_map
    t = cuda_tracer(wl, wl.ring_tables, seed, land, amap)
    while t.samples() < wl.spp:
        t.encode(wl.frame)
    g = t.backward(wl.frame, t.tape(), dl)
    image = t.read_pixels()
    t.close()
    return image, g


def oracle_tangent(wl, d: Direction, seed, land=None):
    t = OracleTracer((wl.width, wl.height), W.render_options(wl, wl.spp))
    for k, v in wl.ring_tables.items():
        t.upload_ring_profile(k, v)
    if land is not None:
        t.upload_terrain(land.terrain, land.cells)
        t.upload_albedo_map(land.albedo_map, land.map_extent)
    _, tan = t.tangent(wl.frame, seed, wl.spp, **d.oracle_kwargs())
    return tan / wl.spp


@pytest.fixture(scope="module")
def rings():
    return ring_scene(48, 27, 16)


@pytest.fixture(scope="module")
def rings_backward(rings):
    dl = loss_weights(48, 27, "field")
    _, g = render_and_backward(rings, 0, dl)
    return dl, g


def directions(wl):
    rng = np.random.default_rng(11)
    dense = Direction(ring_tau={0: rng.uniform(-1, 1, wl.ring_tables[0].size).astype(np.float32)})
    out = {
        "C ring": tau_band(wl, 0, 143),
        "B ring": tau_band(wl, 143, 354),
        "Cassini": tau_band(wl, 354, 392),
        "A ring": tau_band(wl, 392, 512),
        "dense tau": dense,
        "ring albedo": ring_albedo_direction(wl, 2),
    }
    for body, name in enumerate(("star a", "star b", "planet", "moon")):
        out[name] = body_direction(wl, body)
    return out


@pytest.mark.parametrize("name", ["C ring", "B ring", "Cassini", "A ring", "dense tau", "ring albedo", "star a",
                                  "star b", "planet", "moon"])
def test_backward_matches_the_oracle_tangent(rings, rings_backward, name):
    """Same samples, same decisions: the CUDA gradient dotted with a
    direction equals the oracle's tangent along it up to float rounding of
    the (atomic) sums."""
    dl, g = rings_backward
    d = directions(rings)[name]
    expected = float((dl.astype(np.float64) * oracle_tangent(rings, d, 0)).sum())
    got = d.dot(g)
    # Directions with cancelling signs are held to the size of their terms.
    scale = max(abs(expected), 0.05 * d.dot(g, absolute=True))
    assert abs(got - expected) <= 2e-3 * scale, (got, expected, scale)
    assert g.dropped == 0


def test_backward_matches_the_oracle_on_the_albedo_map():
    wl, land = terrain_map_scene(32, 18, 8)
    dl = loss_weights(32, 18, "field")
    _, g = render_and_backward(wl, 0, dl, land)
    d = map_direction(land)
    expected = float((dl.astype(np.float64) * oracle_tangent(wl, d, 0, land)).sum())
    assert abs(d.dot(g) - expected) <= 2e-3 * abs(expected), (d.dot(g), expected)
    assert np.count_nonzero(g.albedo_map) > 0


def test_backward_is_repeatable(rings):
    dl = loss_weights(48, 27, "field")
    t = cuda_tracer(rings, rings.ring_tables, 3)
    while t.samples() < rings.spp:
        t.encode(rings.frame)
    tape = t.tape()
    a = t.backward(rings.frame, tape, dl)
    b = t.backward(rings.frame, tape, dl)
    for x, y in ((a.ring_tau, b.ring_tau), (a.body_color, b.body_color), (a.ring_albedo, b.ring_albedo)):
        np.testing.assert_allclose(x, y, rtol=1e-4, atol=1e-9 * float(np.abs(x).max() + 1e-30))


def test_tape_follows_the_history(rings):
    t = cuda_tracer(rings, rings.ring_tables, 5)
    t.update_options(samples_per_frame=8)
    t.encode(rings.frame)
    t.encode(rings.frame)
    tape = t.tape()
    assert (tape.samples, tape.n_ranges, tape.first[0], tape.count[0]) == (16, 1, 5, 16)
    # A changed frame resets the history and the tape.
    moved = rings.frame.copy()
    moved.scene_time += 1.0
    with pytest.raises(StargazeError) as err:
        t.backward(moved, tape, loss_weights(48, 27))
    assert err.value.status == abi.SG_ERR_STATE
    t.encode(moved)
    tape2 = t.tape()
    assert (tape2.samples, tape2.first[0], tape2.count[0]) == (8, 21, 8)
    # A restored accumulation cannot be replayed.
    t.set_accumulation(t.read_pixels(), 8, 100)
    with pytest.raises(StargazeError) as err:
        t.tape()
    assert err.value.status == abi.SG_ERR_STATE


def test_backward_rejects_bad_arguments(rings):
    t = cuda_tracer(rings, rings.ring_tables, 0)
    t.encode(rings.frame)
    tape = t.tape()
    lib = t._lib
    view = rings.frame.view()
    g = abi.Gradients()
    dl = loss_weights(48, 27)
    assert lib.sg_backward(t.handle, C.byref(view), None, C.c_void_p(dl.ctypes.data), 0, C.byref(g), None) == \
        abi.SG_ERR_INVALID
    bad = abi.Tape.from_buffer_copy(tape)
    bad.count[0] += 1
    assert lib.sg_backward(t.handle, C.byref(view), C.byref(bad), C.c_void_p(dl.ctypes.data), 0, C.byref(g),
                           None) == abi.SG_ERR_INVALID
    t.upload_ring_profile(0, rings.ring_tables[0])  # bumps the history key
    assert lib.sg_backward(t.handle, C.byref(view), C.byref(tape), C.c_void_p(dl.ctypes.data), 0, C.byref(g),
                           None) == abi.SG_ERR_STATE


def cuda_image(wl, frame, tables, seed, land=None, albedo_map=None):
    t = cuda_tracer(wl, tables, seed, land, albedo_map)
    while t.samples() < wl.spp:
        t.encode(frame)
    image = t.read_pixels().astype(np.float64)
    t.close()
    return image


@pytest.mark.parametrize("name", ["A ring", "Cassini", "B ring", "ring albedo", "planet", "star a"])
def test_backward_matches_central_differences(name):
    """Unbiasedness at scale: 256x144, 64 spp, 24 noise batches; the adjoint
    and the central difference of the CUDA forward (h = 2 %, common random
    numbers) agree within four standard errors plus 5 %."""
    wl = ring_scene(256, 144, 64)
    d = directions(wl)[name]
    dl = loss_weights(256, 144)
    fp, tp, _ = apply(wl.frame, wl.ring_tables, None, d, 0.02)
    fm, tm, _ = apply(wl.frame, wl.ring_tables, None, d, -0.02)
    adj, fd = [], []
    for b in range(24):
        seed = 104729 * b
        _, g = render_and_backward(wl, seed, dl)
        adj.append(d.dot(g))
        fd.append(float((dl * (cuda_image(wl, fp, tp, seed) - cuda_image(wl, fm, tm, seed))).sum()) / 0.04)
    adj, fd = np.array(adj), np.array(fd)
    sigma = np.hypot(adj.std(ddof=1), fd.std(ddof=1)) / np.sqrt(len(adj))
    assert abs(adj.mean() - fd.mean()) <= 4.0 * sigma + 0.05 * abs(adj.mean()), (adj.mean(), fd.mean(), sigma)
