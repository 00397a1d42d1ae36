"""The adjoint's checker: the oracle's forward-mode tangent of the
detached-sampling estimator (oracle_tangent) against central differences
of the oracle's forward render with common random numbers.

Parameters that no sampling decision reads (emitted radiance) must match
to rounding; the others (optical depths, albedos) change Russian-roulette
and null-crossing decisions, so their differences are noisy and are
compared over independent noise batches, within four combined standard
errors plus a 2 % margin.
"""
import numpy as np
import pytest

from adjoint_cases import (Direction, apply, body_direction, loss_weights, map_direction, ring_albedo_direction,
                           ring_scene, tau_band, terrain_map_scene)
from oracle.binding import OracleTracer
from stargaze_b200 import workloads as W

WIDTH, HEIGHT, SPP = 48, 27, 32


def oracle_tracer(wl, tables, seed, land=None, albedo_map=None):
    t = OracleTracer((wl.width, wl.height), W.render_options(wl, wl.spp, noise_seed=seed))
    for k, v in tables.items():
        t.upload_ring_profile(k, v)
    if land is not None:
        t.upload_terrain(land.terrain, land.cells)
        if albedo_map is not None:
            t.upload_albedo_map(albedo_map, land.map_extent)
    return t


def render(wl, frame, tables, seed, land=None, albedo_map=None):
    t = oracle_tracer(wl, tables, seed, land, albedo_map)
    t.encode(frame)
    return t.read_pixels().astype(np.float64)


def tangent(wl, d: Direction, seed, land=None):
    t = oracle_tracer(wl, wl.ring_tables, 0, land, None if land is None else land.albedo_map)
    primal, tan = t.tangent(wl.frame, seed, wl.spp, **d.oracle_kwargs())
    return primal, tan / wl.spp


def compare(wl, d: Direction, h: float, batches: int, dl, land=None):
    """Per-batch directional derivatives of sum(dl * image): tangent and
    central difference (same noise keys on both sides)."""
    amap = None if land is None else land.albedo_map
    fp, tp, mp = apply(wl.frame, wl.ring_tables, amap, d, h)
    fm, tm, mm = apply(wl.frame, wl.ring_tables, amap, d, -h)
    tangents, diffs = [], []
    for b in range(batches):
        seed = 7919 * b
        _, tan = tangent(wl, d, seed, land)
        tangents.append(float((dl * tan).sum()))
        plus = (dl * render(wl, fp, tp, seed, land, mp)).sum()
        minus = (dl * render(wl, fm, tm, seed, land, mm)).sum()
        diffs.append(float(plus - minus) / (2.0 * h))
    return np.array(tangents), np.array(diffs)


def assert_agree(tangents, diffs, margin=0.02):
    t, f = tangents.mean(), diffs.mean()
    n = len(tangents)
    sigma = np.hypot(tangents.std(ddof=1), diffs.std(ddof=1)) / np.sqrt(n) if n > 1 else 0.0
    assert abs(t - f) <= 4.0 * sigma + margin * abs(t), (t, f, sigma)


@pytest.fixture(scope="module")
def rings():
    return ring_scene(WIDTH, HEIGHT, SPP)


def test_tangent_primal_is_the_forward_image(rings):
    image = render(rings, rings.frame, rings.ring_tables, 0)
    primal, tan = tangent(rings, Direction(), 0)
    np.testing.assert_array_equal((primal / np.float32(SPP)).astype(np.float32), image.astype(np.float32))
    assert not tan.any()


def test_emitted_radiance_tangent_is_exact(rings):
    """Star radiance reaches no sampling decision: differences and tangent
    agree to rounding on the same samples."""
    dl = loss_weights(WIDTH, HEIGHT, "field")
    for star in (0, 1):
        d = body_direction(rings, star)
        t, f = compare(rings, d, 1e-3, 1, dl)
        assert abs(t[0] - f[0]) <= 1e-3 * abs(t[0]), (star, t, f)


@pytest.mark.parametrize("body", [2, 3])
def test_albedo_tangents(rings, body):
    dl = loss_weights(WIDTH, HEIGHT)
    t, f = compare(rings, body_direction(rings, body), 0.01, 8, dl)
    assert_agree(t, f, 0.005)


def test_ring_albedo_tangent(rings):
    dl = loss_weights(WIDTH, HEIGHT)
    t, f = compare(rings, ring_albedo_direction(rings, 2), 0.01, 8, dl)
    assert_agree(t, f, 0.005)


@pytest.mark.parametrize("band", [(0, 143), (143, 354)], ids=["C ring", "B ring"])
def test_optical_depth_tangents(rings, band):
    """Optical depths move the null/scatter decisions: the tangent must
    still be the derivative of the expected (capped) image."""
    dl = loss_weights(WIDTH, HEIGHT)
    t, f = compare(rings, tau_band(rings, *band), 0.01, 32, dl)
    assert_agree(t, f)


@pytest.mark.parametrize("band", [(354, 392), (392, 512)], ids=["Cassini", "A ring"])
def test_optical_depth_tangents_through_the_ring_cap(band):
    """Enough samples to resolve the ring-indirect cap's share: holding the
    sampling of clamped paths fixed (no likelihood-ratio term) leaves the
    A-ring derivative about 7 % low, outside this tolerance."""
    wl = ring_scene(64, 36, 64)
    dl = loss_weights(64, 36)
    t, f = compare(wl, tau_band(wl, *band), 0.02, 96, dl)
    assert_agree(t, f, 0.01)


def test_albedo_map_tangent():
    wl, land = terrain_map_scene(32, 18, 8)
    dl = loss_weights(32, 18, "field")
    t, f = compare(wl, map_direction(land), 0.01, 4, dl, land)
    assert_agree(t, f, 0.005)
