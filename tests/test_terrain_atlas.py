"""The basalt elevation atlas builder (stargaze_b200.terrain.volcano_atlas)
against the layout volcano.wgsl reads and the reference's own checks of it
(src/volcano.rs:139-170, `elevation_atlas_is_finite_bounded_...`), on
synthetic elevations (the reference's are surveys)."""
import numpy as np

from stargaze_b200.terrain import elevation_pyramid, volcano_atlas


def pyramid_len(width: int) -> int:
    count = width * width
    while width > 1:
        width = (width + 1) // 2
        count += width * width
    return count


def synthetic_maps():
    rng = np.random.default_rng(7)
    return [(rng.uniform(0.0, 900.0, (w, w)).astype(np.float32), s, n)
            for w, s, n in ((65, 5.0, 0.0), (33, 1.0, 250.0), (49, 25.0, 0.0), (17, 25.0, 0.0))]


def test_atlas_layout_matches_the_reference_checks():
    maps = synthetic_maps()
    atlas = volcano_atlas(maps, [(100.0, 200.0, 0.3, 1.2, 2), (-50.0, 10.0, -0.2, 0.9, 3)])
    assert np.isfinite(atlas).all()
    end = 4 * 4 + 9 * 8
    for k, (grid, spacing, north) in enumerate(maps):
        desc = atlas[4 * k:4 * k + 4]
        assert int(desc[0]) == end and int(desc[1]) == grid.shape[0]
        assert desc[2] == np.float32(spacing) and desc[3] == np.float32(north)
        count = pyramid_len(grid.shape[0])
        block = atlas[end:end + count]
        w = grid.shape[0]
        assert np.array_equal(block[:w * w], grid.ravel())
        assert np.all((block >= 0.0) & (block < 1200.0))
        # Every averaged mip stays within its source's range.
        assert np.all(block[w * w:] <= grid.max())
        end += count
    assert end == atlas.size
    # Site 0 is the identity on map 0; the others carry their transforms.
    assert np.array_equal(atlas[16:24], np.array([0, 0, 1, 0, 1, 0, 0, 0], np.float32))
    assert atlas[24 + 4] == np.float32(1.2) and atlas[24 + 5] == 2.0


def test_pyramid_levels_average_with_repeated_odd_edges():
    grid = np.arange(25, dtype=np.float32).reshape(5, 5)
    p = elevation_pyramid(grid)
    assert p.size == 25 + 9 + 4 + 1
    level1 = p[25:34].reshape(3, 3)
    assert level1[0, 0] == np.float32(0.25) * (0 + 1 + 5 + 6)
    # The last column repeats the odd edge sample: (4, 4, 9, 9) / 4.
    assert level1[0, 2] == np.float32(0.25) * (4 + 4 + 9 + 9)
    assert level1[2, 2] == grid[4, 4]
