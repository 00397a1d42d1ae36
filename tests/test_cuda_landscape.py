"""Landscape known answers against the CUDA library (B200)."""
import numpy as np
import pytest

import known_answers as ka
from stargaze_b200 import PathTracer
from stargaze_b200 import terrain as T

pytestmark = pytest.mark.gpu


def make(dimensions, options):
    return PathTracer(dimensions, options)


def test_local_ground_shadows():
    ka.local_ground_shadows(make)


@pytest.mark.parametrize("cells", [128, 512])
def test_heightfield_matches_exhaustive_scan(cells):
    heights = T.fbm_heights(cells, seed=3)
    heights -= heights[(cells + 1) * (cells // 2) + cells // 2]
    ka.heightfield_oracle(make, heights, T.pack_terrain(heights, cells), cells)


def test_heightfield_compact_layout_4096():
    """The extended 4096-cell grid (34-entry traversal stack, compact cache)."""
    cells = 4096
    heights = T.fbm_heights(cells, seed=5)
    rays = [ka.HEIGHTFIELD_RAYS[i] for i in (0, 2, 6)]
    ka.heightfield_oracle(make, heights, T.pack_terrain(heights, cells), cells, rays=rays)


@pytest.mark.parametrize("theme", [0, 3], ids=["forest", "alpine"])
def test_terrain_probe_matches_oracle_bit_exact(theme):
    """Distances bit-exact; normals within 2e-6 (alpine ground mixes the
    smooth normal with the triangle's flat face, terrain.wgsl:142-150)."""
    from oracle.binding import OracleTracer

    cells = 256
    heights = T.fbm_heights(cells, seed=9)
    data = T.pack_terrain(heights, cells)
    rng = np.random.default_rng(4)
    o = np.stack([rng.uniform(-9000, 9000, 512), rng.uniform(0.5, 400, 512), rng.uniform(-9000, 9000, 512)], axis=1)
    d = rng.normal(size=(512, 3))
    d[:, 1] = -np.abs(d[:, 1])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    results = []
    for tracer in (PathTracer((1, 1), ka.test_options()), OracleTracer((1, 1), ka.test_options())):
        tracer.upload_terrain(data, cells)
        f = ka.terrain_frame(6_371_000.0)
        f.globals.ground_counts[2] = (f.globals.ground_counts[2] & ~255) | theme
        results.append(tracer.terrain_probe(f, o.astype(np.float32), d.astype(np.float32)))
    cuda, cpu = results
    assert np.array_equal(cuda[:, 3], cpu[:, 3])  # distances bit-exact (and misses)
    hit = cpu[:, 3] < 1e29
    assert hit.mean() > 0.5
    assert np.abs(cuda[hit, :3] - cpu[hit, :3]).max() < 2e-6
