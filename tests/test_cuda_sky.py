"""The camera-only sky backdrop (sg_upload_catalogue, sg_upload_milky_way;
pathtrace.wgsl:268-334, :1494-1508) against the oracle on the same uploaded
tables: catalogue discs seen through a telescope field, the Milky Way seen
past a ringed planet (through its ring's transmission), both integrators,
the accumulation and the separate backdrop accumulation. Bar: the parity
bar of test_cuda_parity.py (2e-3 relative RMSE, 99 % of pixels within 1e-4
relative); the CUDA and C library arc functions may differ by an ulp."""
import numpy as np
import pytest

import golden_io as gio
import known_answers as ka
from oracle.binding import OracleTracer
from stargaze_b200 import sky
from stargaze_b200._lib import StargazeError
from stargaze_b200.pathtracer import PathTracer
from stargaze_b200.scene import body, frame, ringed

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables():
    stars, cells = sky.ray_catalogue(sky.generate(3500, 2500, 0x5EED1234))
    return stars, cells, sky.panorama()


def basis(forward):
    f = np.asarray(forward, np.float64)
    f /= np.linalg.norm(f)
    r = np.cross(f, [0.0, 0.0, 1.0])
    r /= np.linalg.norm(r)
    return r, np.cross(r, f), f


def view_frame(forward, tan_half, size):
    f = frame()
    r, u, fw = basis(forward)
    f.globals.cam_right[:] = [*r, 0.0]
    f.globals.cam_up[:] = [*u, 0.0]
    f.globals.cam_forward[:] = [*fw, tan_half]
    f.globals.viewport[:] = [float(size[0]), float(size[1]), 1.0, size[0] / size[1]]
    return f


def telescope_frame(stars, size):
    """A 0.5-degree field centred on the catalogue's brightest star."""
    k = int(np.argmax(stars[:, 4:7].sum(axis=1)))
    return view_frame(stars[k, :3], 0.004, size)


def galactic_frame(size):
    """A 60-degree field in the galactic plane, a ringed planet in front
    (telescope-space centre along the view, so its ring crosses the band)."""
    pole = np.array(sky.GALACTIC_POLE) / np.linalg.norm(sky.GALACTIC_POLE)
    d = np.cross(pole, [1.0, 0.0, 0.0])
    f = view_frame(d, 0.6, size)
    f.bodies = [body([0.3, -0.2, -12.0], 1.0, [0.4, 0.4, 0.4], False),
                body([40.0, 10.0, 30.0], 0.5, [30.0, 30.0, 30.0], True)]
    f.bodies[0] = ringed([0.3, -0.2, -12.0], 1.0, [0.2, 0.9, 0.4], 0.7)
    f.bodies[0].color[:] = [0.4, 0.4, 0.4]
    return f


def render_pair(f, size, tables, integrator, milky=4.0e-4, spp=8):
    stars, cells, pano = tables
    opts = ka.test_options(samples_per_frame=spp, max_bounces=4, milky_way=milky)
    g = PathTracer(size, opts)
    o = OracleTracer(size, opts)
    g.set_integrator(integrator)
    for t in (g, o):
        t.upload_catalogue(stars, cells)
        t.upload_milky_way(pano)
        t.encode(f)
        t.encode(f)
    out = (g.read_pixels(), o.read_pixels(), g.read_backdrop(), o.read_backdrop())
    g.close()
    return out


def assert_parity(img, ref):
    assert np.isfinite(img).all()
    assert gio.relative_rmse(img, ref) < 2e-3
    close = np.abs(img[:, :3] - ref[:, :3]) <= 1e-4 * np.maximum(np.abs(ref[:, :3]), 1e-3 * np.abs(ref[:, :3]).max())
    assert close.all(axis=1).mean() >= 0.99


@pytest.mark.parametrize("integrator", ["wavefront", "megakernel"])
def test_catalogue_discs_through_a_telescope(tables, integrator):
    size = (48, 32)
    f = telescope_frame(tables[0], size)
    img, ref, _, _ = render_pair(f, size, tables, integrator, milky=0.0)
    assert ref[:, :3].max() > 0, "the brightest star lies in the field"
    assert_parity(img, ref)
    np.testing.assert_array_equal(img[:, 3], 0.0)  # no Milky Way: no backdrop luminance


@pytest.mark.parametrize("integrator", ["wavefront", "megakernel"])
def test_milky_way_behind_a_ringed_planet(tables, integrator):
    size = (64, 48)
    f = galactic_frame(size)
    img, ref, bd, bref = render_pair(f, size, tables, integrator)
    assert bref[:, :3].max() > 0
    assert_parity(img, ref)
    np.testing.assert_allclose(img[:, 3], ref[:, 3], rtol=1e-4, atol=1e-4 * float(ref[:, 3].max()))
    np.testing.assert_allclose(bd[:, :3], bref[:, :3], rtol=1e-4, atol=1e-4 * float(bref[:, :3].max()))
    # The backdrop is part of the image and its luminance is the w channel.
    np.testing.assert_allclose(img[:, 3], bd[:, :3] @ np.array([0.2126, 0.7152, 0.0722]), rtol=1e-5,
                               atol=1e-6 * float(img[:, 3].max()))


def test_removing_the_sky_clears_the_backdrop(tables):
    size = (32, 24)
    f = galactic_frame(size)
    stars, cells, pano = tables
    t = PathTracer(size, ka.test_options(samples_per_frame=4, max_bounces=4, milky_way=4.0e-4))
    t.upload_milky_way(pano)
    t.encode(f)
    assert t.read_backdrop()[:, :3].max() > 0
    t.upload_milky_way(None)
    t.encode(f)
    assert t.samples() == 4
    np.testing.assert_array_equal(t.read_backdrop(), 0.0)
    np.testing.assert_array_equal(t.read_pixels()[:, 3], 0.0)
    t.close()


def test_backward_rejects_a_sky(tables):
    size = (16, 16)
    f = galactic_frame(size)
    t = PathTracer(size, ka.test_options(samples_per_frame=4, max_bounces=4, milky_way=4.0e-4))
    t.upload_milky_way(tables[2])
    t.encode(f)
    with pytest.raises(StargazeError):
        t.backward(f, t.tape(), np.ones((16 * 16, 4), np.float32))
    t.close()
