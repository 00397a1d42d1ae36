"""Landscape known answers against the CPU oracle (no GPU)."""
import numpy as np
import pytest

import known_answers as ka
from oracle.binding import OracleTracer
from stargaze_b200 import terrain as T


def make(dimensions, options):
    return OracleTracer(dimensions, options)


def test_local_ground_shadows():
    r = ka.local_ground_shadows(make)
    assert set(r) == {6_371_000.0, 1_500_000.0}


@pytest.mark.parametrize("cells", [128, 512])
def test_heightfield_matches_exhaustive_scan(cells):
    heights = T.fbm_heights(cells, seed=3)
    heights -= heights[(cells + 1) * (cells // 2) + cells // 2]  # ground at the observer
    data = T.pack_terrain(heights, cells)
    results = ka.heightfield_oracle(make, heights, data, cells)
    hits = [r for r in results if np.isfinite(r[3])]
    assert len(hits) >= 10  # most rays hit; misses are checked too


def test_heightfield_compact_layout():
    """Grids over 1024 cells use the compact vertex cache (12+12-bit
    normals, no derivatives): a 2048-cell grid on three rays."""
    cells = 2048
    heights = T.fbm_heights(cells, seed=5)
    data = T.pack_terrain(heights, cells)
    assert data.size == T.bounds_offset(cells) + 2 * T.node_count(cells)
    rays = [ka.HEIGHTFIELD_RAYS[i] for i in (0, 2, 6)]
    ka.heightfield_oracle(make, heights, data, cells, rays=rays)


def test_pack_terrain_bounds_are_conservative():
    cells = 64
    h = T.fbm_heights(cells, seed=1)
    d = T.pack_terrain(h, cells)
    off = T.bounds_offset(cells)
    H = h.reshape(cells + 1, cells + 1)
    # Root bounds cover every vertex; a child's bounds lie inside its parent's.
    assert d[off] == H.min() and d[off + 1] == H.max()
    for node in range(1, T.node_count(cells)):
        parent = (node - 1) // 4
        assert d[off + 2 * parent] <= d[off + 2 * node] <= d[off + 2 * node + 1] <= d[off + 2 * parent + 1]


def test_prop_bvh_groups_every_prop_once():
    rng = np.random.default_rng(0)
    props = [T.primitive(rng.uniform(-50, 50, 3), 1.0, rng.uniform(0.2, 2, 3), 0.0, (0.3, 0.4, 0.2), 0.0)
             for _ in range(300)]
    flat = T.build_prop_bvh(props, leaf_size=4)
    leaves = [p for p in flat if p.center[3] >= 0]
    assert len(leaves) == 300
    # Every marker's skip stays inside the list and covers its children.
    for i, p in enumerate(flat):
        if p.center[3] < 0:
            skip = int(-p.center[3])
            assert i + skip < len(flat)
            lo = np.array(p.center[:3]) - np.array(p.extent[:3])
            hi = np.array(p.center[:3]) + np.array(p.extent[:3])
            for q in flat[i + 1: i + 1 + skip]:
                if q.center[3] >= 0:
                    c = np.array(q.center[:3])
                    assert np.all(c >= lo) and np.all(c <= hi)
