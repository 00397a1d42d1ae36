"""The oracle reproduces the committed golden fixtures (no GPU)."""
import numpy as np
import pytest

import golden_io as gio
from golden.make_golden import IMAGES, image_fixture, landscape_of, make_tracer, scenes


@pytest.mark.parametrize("name", gio.RAY_SCENES)
def test_oracle_reproduces_ray_fixtures(name):
    f, tables = scenes()[name]
    g = gio.load_rays(name)
    t = make_tracer(f, tables, land=landscape_of(name))
    hits = t.closest_hit(f, g["rays"])
    assert np.array_equal(hits["index"], g["hit_index"])
    assert np.array_equal(hits["distance"], g["hit_distance"])
    assert np.array_equal(hits["normal"], g["hit_normal"])
    vis = t.light_visibility(f, g["vis_rays"], g["vis_lights"])
    assert np.array_equal(vis, g["visibility"])
    for i in range(len(f.bodies)):
        assert np.array_equal(t.ring_probe(f, g["rays"], i), g["ring"][i])


@pytest.mark.parametrize("name", gio.IMAGE_NAMES)
def test_oracle_reproduces_image_fixtures(name):
    assert name in IMAGES
    img = image_fixture(name)
    assert np.array_equal(img, gio.load_image(name))


def test_fixtures_are_not_degenerate():
    for name in gio.RAY_SCENES:
        g = gio.load_rays(name)
        hit = g["hit_index"] != 0xFFFFFFFF
        assert 0.1 < hit.mean() < 0.9, name
        assert (g["visibility"] > 0).mean() > 0.05, name
    for name in gio.IMAGE_NAMES:
        img = gio.load_image(name)
        assert np.isfinite(img).all() and (img >= 0).all()
        assert (img[:, :3].sum(axis=1) > 0).mean() > 0.05, name


def test_terrain_fixture_exercises_every_landscape_kind():
    g = gio.load_rays("terrain")
    idx = g["hit_index"]
    assert (idx == 0x80000000).sum() > 0 or (idx == 0x80100000).sum() > 0  # ground
    assert (idx == 0x80100000).sum() > 100  # terrain
    assert ((idx > 0x80000000) & (idx < 0x80100000)).sum() > 20  # props
