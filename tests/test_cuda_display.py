"""sg_display and the automatic exposure of sg_encode against the display
oracle (oracle/display.py), which test_oracle_display.py pins to the
reference's known answers. Bar: linear output within 1e-5 of the oracle
(the reference's own tolerance for its Rgba32Float display tests), sRGB
bytes within one code of it."""
import numpy as np
import pytest

import known_answers as ka
from oracle import display as D
from stargaze_b200.headless import capture, read_png_rgba
from stargaze_b200.pathtracer import PathTracer
from stargaze_b200.scene import body, frame

pytestmark = pytest.mark.gpu

COLORS = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [1, 1, 1, 0]], np.float32)


def tracer_with(accumulation, size, **options):
    t = PathTracer(size, ka.test_options(**options))
    t.set_accumulation(accumulation, 1, 1)
    return t


@pytest.mark.parametrize("out", [(4, 4), (2, 2), (1, 1)])
def test_upscale_matches_the_reference_test(out):
    t = tracer_with(COLORS, (2, 2))
    got = t.display(out, linear=True)
    t.close()
    ref = D.display(COLORS, 2, 2, out[0], out[1], exposure=1.0)
    np.testing.assert_allclose(got[..., :3], ref, atol=1e-5)
    np.testing.assert_array_equal(got[..., 3], 1.0)


@pytest.mark.parametrize("out", [(37, 23), (64, 40), (20, 12), (1, 1)])
def test_random_hdr_linear_and_srgb(out):
    rng = np.random.default_rng(4)
    acc = np.zeros((23 * 37, 4), np.float32)
    acc[:, :3] = np.exp(rng.uniform(np.log(1e-4), np.log(1e3), (23 * 37, 3)))
    t = tracer_with(acc, (37, 23), exposure=0.3, ev_bias=0.5)
    lin = t.display(out, linear=True)
    srgb = t.display(out)
    t.close()
    ref = D.display(acc, 37, 23, out[0], out[1], exposure=0.3, bias=0.5)
    np.testing.assert_allclose(lin[..., :3], ref, atol=1e-5)
    diff = np.abs(srgb[..., :3].astype(np.int32) - D.srgb8(ref).astype(np.int32))
    assert diff.max() <= 1, diff.max()
    np.testing.assert_array_equal(srgb[..., 3], 255)


@pytest.mark.parametrize("base,bias,expected", [(1.0, 80.0, 1.0), (1.0, -1000.0, 0.0), (1.0, 1000.0, 1.0),
                                                (float(np.finfo(np.float32).max), 0.0, 1.0)])
def test_extreme_exposure_controls(base, bias, expected):
    star = np.array([[10.0, 10.0, 10.0, 0.0]], np.float32)
    t = tracer_with(star, (1, 1), exposure=base, ev_bias=bias)
    got = t.display(linear=True)
    t.close()
    assert np.isfinite(got).all()
    np.testing.assert_allclose(got[0, 0, :3], expected, atol=1e-5)


def star_frame():
    f = frame()
    f.bodies = [body([0.0, 0.0, -3.0], 1.0, [10.0] * 3, True)]
    return f


def test_auto_exposure_meters_a_single_pixel():
    """ring_tests.rs:454-477: 64 one-sample encodes of a star filling a
    one-pixel viewport ease the exposure to 0.25 / 10 within 10 %; the value
    equals the oracle's easing of the same accumulation."""
    t = PathTracer((1, 1), ka.test_options(auto_exposure=1))
    f = star_frame()
    for _ in range(64):
        t.encode(f)
    acc = t.read_pixels()
    value = t.exposure()
    t.close()
    np.testing.assert_allclose(acc[0, :3], 10.0, rtol=1e-6)
    assert abs(value / 0.025 - 1.0) < 0.1, value
    ref = D.eased_exposure(acc, 1, 1, start=1.0, key=0.25, percentile=0.9, encodes=64)
    np.testing.assert_allclose(value, ref, rtol=1e-4)


def test_auto_exposure_keeps_metering_after_convergence():
    """ring_tests.rs:479-503: once the sample limit is reached, encodes add
    no sample but still meter; the image does not change."""
    t = PathTracer((8, 8), ka.test_options(sample_limit=1))
    f = star_frame()
    f.globals.viewport[:2] = [8.0, 8.0]
    t.encode(f)
    before = t.read_pixels()
    t.set_exposure_controls(True, 0.0)
    for _ in range(64):
        t.encode(f)
    after = t.read_pixels()
    value = t.exposure()
    assert t.samples() == 1
    t.close()
    np.testing.assert_array_equal(before, after)
    assert abs(value / 0.025 - 1.0) < 0.1, value


def test_headless_capture_writes_the_display(tmp_path):
    t = PathTracer((32, 24), ka.test_options(samples_per_frame=4))
    f = star_frame()
    f.globals.viewport[:2] = [32.0, 24.0]
    f.globals.cam_forward[3] = 0.5
    cap = capture(t, f, 8, tmp_path / "out.png")
    png = read_png_rgba(tmp_path / "out.png")
    np.testing.assert_array_equal(png, t.display())
    t.close()
    assert cap["samples"] == 8 and cap["width"] == 32 and cap["height"] == 24
    assert png[..., :3].max() > 0
