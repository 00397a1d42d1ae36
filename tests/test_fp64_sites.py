"""FP64 sites (PathTracer.set_fp64_sites): the host-sphere intersection, the
ring-plane intersection and the 5 mm bounce offset evaluated in double from
the same f32 inputs. The default f32 variant is the reference's arithmetic
and is what every parity test checks; these tests bound the error of both
variants against the exact intersection of the same f32 rays."""
import numpy as np
import pytest

from stargaze_b200 import precision as P
from stargaze_b200 import workloads as W

# The device returns f32 AU distances and f32 radii: one rounding each
# (2^-24 relative) plus the f32 length of the f32 hit point.
FP64_DISTANCE_TOL = 2.5e-7
FP64_RADIUS_TOL = 5e-7


def test_host_sphere_closed_form_lies_on_the_sphere():
    frame = P.host_sphere_frame()
    rays, t, past = P.host_sphere_rays(frame, 20000, seed=5)
    g = frame.globals
    basis = np.array([g.ground_east[:3], g.ground_up[:3], g.ground_north[:3]], np.float64)
    d = rays["direction"].astype(np.float64) @ basis.T
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    h, r = g.ground_east[3], g.ground_up[3]
    point = d * t[:, None] + np.array([0.0, r + h, 0.0])
    np.testing.assert_allclose(np.linalg.norm(point, axis=1), r, rtol=1e-12)
    assert np.isfinite(t).all() and (t > 0).all() and past.min() >= 1e-6 * 0.999


def test_ring_closed_form_lies_in_the_plane():
    wl = W.rings_1080p(64, 64, 1)
    (body,) = P.ring_bodies(wl.frame)
    rays, t, r, inside = P.ring_rays(wl.frame, body, 20000, seed=5)
    b = wl.frame.bodies[body]
    centre = np.array(b.center[:], np.float64) + np.array(b.center_low[:3], np.float64)
    pole = np.array(b.ring_plane[:3], np.float32).astype(np.float64)
    point = rays["direction"].astype(np.float64) * t[:, None] - centre
    assert np.abs(point @ pole).max() < 1e-12 * np.abs(t).max()
    assert inside.mean() > 0.99


@pytest.mark.gpu
def test_host_sphere_fp64_sites_are_exact_to_f32_rounding():
    f32 = P.host_sphere_precision(10**6, fp64=False, seed=1)
    fp64 = P.host_sphere_precision(10**6, fp64=True, seed=1)
    for m in (f32, fp64):
        assert m["hits_found"] == m["hits_expected"] == 10**6
    assert fp64["relative_error"]["max"] < FP64_DISTANCE_TOL, fp64
    # The reference's f32 quadratic: a few 1e-5 beyond 1 mrad past the
    # horizon dip, up to ~1e-3 when grazing.
    assert f32["relative_error_beyond_1mrad"] < 1e-4, f32
    assert f32["relative_error"]["max"] < 5e-3, f32
    assert f32["relative_error"]["max"] > 10 * fp64["relative_error"]["max"]


@pytest.mark.gpu
def test_ring_plane_fp64_sites_are_exact_to_f32_rounding():
    wl = W.rings_1080p(64, 64, 1)
    f32 = P.ring_plane_precision(wl.frame, 10**6, fp64=False, tables=wl.ring_tables, seed=2)
    fp64 = P.ring_plane_precision(wl.frame, 10**6, fp64=True, tables=wl.ring_tables, seed=2)
    for body, m in fp64.items():
        assert m["hits_found"] == m["hits_expected"], m
        assert m["distance_relative_error"]["max"] < FP64_DISTANCE_TOL, m
        assert m["radius_relative_error"]["max"] < FP64_RADIUS_TOL, m
        assert f32[body]["hits_found"] >= 0.999 * f32[body]["hits_expected"]
        assert f32[body]["radius_relative_error"]["max"] < 1e-3, f32[body]


def _render(wl, fp64: bool):
    from stargaze_b200.pathtracer import PathTracer

    t = PathTracer((wl.width, wl.height), W.render_options(wl, wl.spp, noise_seed=3))
    W.upload_workload(t, wl)
    t.set_fp64_sites(fp64)
    frame = wl.frame.copy()
    while t.samples() < wl.spp:
        t.encode(frame)
    image = t.read_pixels()[:, :3].astype(np.float64)
    t.close()
    return image


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["rings", "terrain"])
def test_fp64_sites_render_the_same_image(scene):
    """Same noise sequence, same scene: the two variants differ only where a
    path's hit moves by float rounding, so the images agree closely."""
    if scene == "rings":
        wl = W.rings_1080p(96, 64, 16)
    else:
        wl, _ = W.terrain_1080p(96, 64, 16, cells=256, rocks=50, foliage=50)
    a, b = _render(wl, False), _render(wl, True)
    assert a.sum() > 0
    rel = np.sqrt(((a - b) ** 2).sum() / (a ** 2).sum())
    assert rel < 0.02, rel
