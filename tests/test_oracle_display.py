"""The display oracle (oracle/display.py) pinned to the reference's own
known answers for the display pass and the automatic exposure:
pathtracer_tests.rs:316-430 (upscale, orientation and edges),
pathtracer_tests.rs:1266-1359 (extreme exposure controls),
ring_tests.rs:454-477 (single-pixel metering) and the metered region of
pathtracer.rs:40-42."""
import numpy as np
import pytest

from oracle import display as D

COLORS = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [1, 1, 1, 0]], np.float32)


@pytest.mark.parametrize("size", [(4, 4), (2, 2), (1, 1)])
def test_upscale_keeps_orientation_and_edges(size):
    w, h = size
    out = D.display(COLORS, 2, 2, w, h, exposure=1.0)
    aces = D.aces
    if w == 1:
        np.testing.assert_allclose(out[0, 0], aces([0.5] * 3), atol=1e-5)
        return
    np.testing.assert_allclose(out[0, 0], aces([1, 0, 0]), atol=1e-5)
    np.testing.assert_allclose(out[0, w - 1], aces([0, 1, 0]), atol=1e-5)
    np.testing.assert_allclose(out[h - 1, 0], aces([0, 0, 1]), atol=1e-5)
    np.testing.assert_allclose(out[h - 1, w - 1], aces([1, 1, 1]), atol=1e-5)
    if w == 4:
        np.testing.assert_allclose(out[1, 1], aces([0.625, 0.25, 0.25]), atol=1e-5)


@pytest.mark.parametrize("base,bias,expected", [(1.0, 80.0, 1.0), (1.0, -1000.0, 0.0), (1.0, 1000.0, 1.0),
                                                (float(np.finfo(np.float32).max), 0.0, 1.0)])
def test_extreme_exposure_controls_stay_finite(base, bias, expected):
    star = np.array([[10.0, 10.0, 10.0, 0.0]], np.float32)
    out = D.display(star, 1, 1, 1, 1, exposure=base, bias=bias)
    assert np.isfinite(out).all()
    np.testing.assert_allclose(out[0, 0], expected, atol=1e-5)


def test_single_pixel_metering_targets_the_key():
    """A one-pixel viewport of radiance 10 eases to 0.25 / 10 within 10 %
    after 64 meterings (one per encode of one sample)."""
    star = np.array([[10.0, 10.0, 10.0, 0.0]], np.float32)
    value = D.eased_exposure(star, 1, 1, start=1.0, key=0.25, percentile=0.9, encodes=64)
    assert abs(value / 0.025 - 1.0) < 0.1, value


@pytest.mark.parametrize("size,region", [((1, 1), (0, 0, 1, 1)), ((5, 3), (1, 0, 3, 3)),
                                         ((160, 90), (40, 22, 80, 46)), ((8, 8), (2, 2, 4, 4))])
def test_meter_region_matches_the_shader(size, region):
    assert D.meter_region(*size) == region


def test_empty_histogram_keeps_the_exposure():
    assert D.resolve(np.zeros(D.BINS, np.int64), 0.7, 0.25, 0.9) == 0.7


def test_dark_and_invalid_pixels_fall_into_the_first_bin():
    img = np.array([[0, 0, 0, 0], [np.nan, 0, 0, 0], [1, 1, 1, 5.0], [1e-30, 0, 0, 0]], np.float32)
    hist = D.histogram(img, 2, 2)  # a 2x2 viewport is metered whole
    assert hist[0] == 4
    hist = D.histogram(img, 4, 1)  # x = 1, 2: NaN, and luminance below the backdrop
    assert hist.sum() == 2 and hist[0] == 2


def test_srgb_encoding():
    np.testing.assert_array_equal(D.srgb8([0.0, 1.0, 0.5, 0.0031308, 0.2]), [0, 255, 188, 10, 124])
