"""The algorithmic-work model's event counts: the counting variant of the
CUDA integrator (sg_encode_counted) against the oracle's counters on the
same frames and noise keys. The roofline's operation count is these events
times a fixed cost per event, so the device must count exactly the work the
reference algorithm does: equal counts, up to the rare path whose decision
flips at an ulp of a transcendental (relative difference 1e-3 at most)."""
import ctypes as C

import numpy as np
import pytest

import known_answers as ka
from golden.make_golden import image_workload
from oracle.binding import Events, OracleTracer
from stargaze_b200 import _lib
from stargaze_b200.pathtracer import PathTracer

pytestmark = pytest.mark.gpu

NAMES = [name for name, _ in Events._fields_ if name != "samples"]


def counted(frame, tables, size, land, spp, bounces):
    opts = ka.test_options(samples_per_frame=spp, max_bounces=bounces)
    gpu = PathTracer(size, opts)
    cpu = OracleTracer(size, opts)
    for t in (gpu, cpu):
        for slot, tau in tables.items():
            t.upload_ring_profile(slot, tau)
        if land is not None:
            t.upload_terrain(land.terrain, land.cells)
    lib = _lib.load()
    ev = (C.c_uint64 * len(NAMES))()
    view = frame.view()
    assert lib.sg_encode_counted(gpu.handle, C.byref(view), None, ev) == 0, lib.sg_last_error(gpu.handle)
    gpu.close()
    cpu.encode(frame)
    return dict(zip(NAMES, list(ev))), cpu.events.as_dict()


@pytest.mark.parametrize("name", ["rings_96x54", "spheres_64", "terrain_96x54"])
def test_counting_kernel_counts_the_oracle_events(name):
    wl, land = image_workload(name)
    size = (96, 54) if name != "spheres_64" else (64, 64)
    got, ref = counted(wl.frame, wl.ring_tables, size, land, 8, wl.max_bounces)
    assert ref["samples"] == size[0] * size[1] * 8
    for key in NAMES:
        r, g = ref[key], got[key]
        assert abs(int(g) - int(r)) <= max(1e-3 * r, 2), (key, g, r)
    if land is not None:
        assert ref["terrain_nodes"] > 0 and ref["terrain_triangles"] > 0 and ref["prop_tests"] > 0
