"""sg_closest_hit_noalloc: closest-hit queries for callers that cannot let
the library allocate device memory (a host application that gives the whole
device to its own allocator or pool, or a latency-bound caller for which
cudaMalloc's device synchronisation is too slow). It stages bodies, rays and
hits in one fixed device array instead of a context's cudaMalloc'd buffer,
and must return exactly what sg_closest_hit returns.

Collected last on purpose: the array is shared by every call in the
process, so the test also shows that earlier work leaves nothing behind
that changes its results.
"""
import ctypes as C

import numpy as np
import pytest

from rays import seeded_rays
from stargaze_b200 import _lib, abi, workloads as W
from stargaze_b200.pathtracer import HIT_DTYPE, PathTracer

pytestmark = pytest.mark.gpu


def noalloc_closest_hit(lib, frame, rays, n=None):
    rays = np.ascontiguousarray(rays)
    hits = np.zeros(len(rays), dtype=HIT_DTYPE)
    view = frame.view()
    status = lib.sg_closest_hit_noalloc(0, C.byref(view), C.c_void_p(rays.ctypes.data),
                                        len(rays) if n is None else n, C.c_void_p(hits.ctypes.data), None)
    return status, hits


def reference_hits(frame, tables, rays):
    t = PathTracer((64, 64))
    for slot, tau in tables.items():
        t.upload_ring_profile(slot, tau)
    hits = t.closest_hit(frame, rays)
    t.close()
    return hits


@pytest.mark.parametrize("scene", ["spheres_256", "rings_1080p"])
def test_noalloc_closest_hit_equals_sg_closest_hit(scene):
    """Two calls in a row (different ray sets, the second larger) give the
    ids and distances of sg_closest_hit bit for bit and its normals within
    the parity tolerance of the closest-hit tests (2e-6)."""
    lib = _lib.load()
    wl = W.WORKLOADS[scene](width=64, height=64)
    for seed, n in ((3, 4096), (4, 20000)):
        rays = seeded_rays(wl.frame, n, seed)
        status, hits = noalloc_closest_hit(lib, wl.frame, rays)
        assert status == abi.SG_OK, lib.sg_last_error(None)
        ref = reference_hits(wl.frame, wl.ring_tables, rays)
        np.testing.assert_array_equal(hits["index"], ref["index"])
        np.testing.assert_array_equal(hits["distance"], ref["distance"])
        np.testing.assert_allclose(hits["normal"], ref["normal"], rtol=0, atol=2e-6)
        assert (hits["index"] != abi.MISS).any()


def test_noalloc_closest_hit_allocates_no_device_memory():
    """After a first call (which loads the kernel and looks up the array's
    address), a call at the largest size leaves the device's free memory
    unchanged."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    wl = W.rings_1080p(width=64, height=64)
    status, _ = noalloc_closest_hit(lib, wl.frame, seeded_rays(wl.frame, 64, 5))
    assert status == abi.SG_OK, lib.sg_last_error(None)
    rays = seeded_rays(wl.frame, abi.NOALLOC_MAX_RAYS, 6)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(0)
    status, hits = noalloc_closest_hit(lib, wl.frame, rays)
    free_after, _ = torch.cuda.mem_get_info(0)
    assert status == abi.SG_OK, lib.sg_last_error(None)
    assert (hits["index"] != abi.MISS).any()
    assert free_after == free_before


def test_noalloc_closest_hit_rejects_what_it_cannot_stage():
    lib = _lib.load()
    wl = W.spheres_256(width=64, height=64)
    rays = seeded_rays(wl.frame, 16, 1)
    status, _ = noalloc_closest_hit(lib, wl.frame, rays, n=abi.NOALLOC_MAX_RAYS + 1)
    assert status == abi.SG_ERR_CAPACITY
    assert b"SG_NOALLOC_MAX_RAYS" in lib.sg_last_error(None)
    land = wl.frame.copy()
    land.globals.ground_north[3] = 2.0
    status, _ = noalloc_closest_hit(lib, land, rays)
    assert status == abi.SG_ERR_INVALID
    assert b"landscape" in lib.sg_last_error(None)
    status, _ = noalloc_closest_hit(lib, wl.frame, rays[:0])
    assert status == abi.SG_OK
