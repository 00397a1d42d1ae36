"""Host-side tables of the sky backdrop (stargaze_b200/sky.py) against the
reference's own unit tests of them: src/stars.rs:207-245 (every sample of
every disc lies in a cell that lists it, across the longitude seam and at
both poles) and src/sky.rs:120-147 (the haze wraps at the seam, vanishes
near the poles, has a broad warm bulge and cool outer clouds)."""
import math

import numpy as np

from stargaze_b200 import sky


def test_grid_contains_disc_samples_including_seam_and_poles():
    stars = sky.generate(100, 0, 123)
    for d in ([-1.0, 0.0, 0.0], [0.0, 0.0, 1.0], [0.0, 0.0, -1.0]):
        stars.append({"dir": d, "color": [1.0, 1.0, 1.0], "angular_radius": 0.0012, "bright": 1.0})
    _, cells = sky.ray_catalogue(stars)
    n_cells = sky.GRID_W * sky.GRID_H
    for i, star in enumerate(stars):
        axis = np.array(star["dir"], np.float64)
        axis /= np.linalg.norm(axis)
        tangent = sky._orthonormal(axis)
        bitangent = np.cross(axis, tangent)
        for j in range(32):
            phi = j * 2.0 * math.pi / 32.0
            radius = float(star["angular_radius"]) * 0.999
            d = axis * math.cos(radius) + (tangent * math.cos(phi) + bitangent * math.sin(phi)) * math.sin(radius)
            x = min(int((math.atan2(d[1], d[0]) + math.pi) / (2.0 * math.pi) * 256.0), 255)
            y = min(int(math.acos(min(max(d[2], -1.0), 1.0)) / math.pi * 128.0), 127)
            cell = y * 256 + x
            start, end = n_cells + 1 + cells[cell], n_cells + 1 + cells[cell + 1]
            assert i in cells[start:end], (i, cell)


def test_catalogue_rows():
    stars = sky.generate(40, 20, 7)
    data, cells = sky.ray_catalogue(stars)
    assert data.shape == (60, 8) and cells.dtype == np.uint32
    np.testing.assert_allclose(np.linalg.norm(data[:, :3], axis=1), 1.0, rtol=1e-6)
    assert (data[:, 3] > 0).all() and (data[:, 3] < 1e-5).all()
    assert (data[:, 4:7] >= 0).all() and (data[:, 4:7].sum(axis=1) > 0).all()
    assert cells[sky.GRID_W * sky.GRID_H] == len(cells) - sky.GRID_W * sky.GRID_H - 1
    # The band stars cluster near the galactic plane.
    pole = np.array(sky.GALACTIC_POLE) / np.linalg.norm(sky.GALACTIC_POLE)
    assert np.abs(data[40:, :3] @ pole).mean() < np.abs(data[:40, :3] @ pole).mean()


def test_haze_wraps_and_has_dust_contrast_without_pole_glow():
    for lat in (-0.2, -0.05, 0.0, 0.05, 0.2):
        left, right = sky.haze_color(-math.pi, lat), sky.haze_color(math.pi, lat)
        assert np.linalg.norm(left - right) < 1e-6
    assert not sky.haze_color(0.0, 1.5).any() and not sky.haze_color(0.0, -1.5).any()
    assert np.linalg.norm(sky.haze_color(0.0, 0.35)) > 2.0 * np.linalg.norm(sky.haze_color(math.pi, 0.35))
    warm, cool = sky.haze_color(0.0, 0.25), sky.haze_color(math.pi, 0.1)
    assert warm[0] > warm[2] and cool[2] > cool[0]


def test_panorama_texels():
    m = sky.panorama()
    assert m.shape == (sky.PANORAMA_H, sky.PANORAMA_W) and m.dtype == np.uint32
    assert (m != 0).any() and (m == 0).any()
    assert ((m & 1023) <= 1023).all() and (m >> 30 == 0).all()
