"""C-ABI checks that need no GPU: layouts, loading, exported symbols."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from stargaze_b200 import _lib, abi

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_symbols() -> set[str]:
    names = set()
    for h in HEADERS:
        for m in re.finditer(r"SG_API\s+[^;(]*?\b(sg_\w+)\s*\(", h.read_text()):
            names.add(m.group(1))
    return names


@pytest.mark.parametrize("name", sorted(abi.LAYOUT_SIZES))
def test_layout_sizes(name):
    cls, size = abi.LAYOUT_SIZES[name]
    assert C.sizeof(cls) == size


def test_layout_offsets_match_the_reference_order():
    # Settings = Globals + counts + sampling + background + lights
    # (src/pathtracer.rs:46-52); Sphere fields in src/renderer.rs:35-48 order.
    assert abi.Settings.counts.offset == 176
    assert abi.Settings.lights.offset == 224
    assert abi.Sphere.center_low.offset == 32
    assert abi.Sphere.ring_plane.offset == 48
    assert abi.Sphere.surface_params.offset == 144
    assert abi.Globals.ground_counts.offset == 160


def test_header_declares_what_the_binding_types():
    assert declared_symbols() == set(_lib.exported_symbols())


def test_library_loads_and_exports_every_declared_symbol(cuda_lib):
    for name in declared_symbols():
        assert hasattr(cuda_lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIBRARY_PATH)], capture_output=True, text=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if " T " in line}
    assert declared_symbols() <= exported
    # Nothing but the C ABI is exported.
    assert {s for s in exported if not s.startswith("sg_")} <= {"_init", "_fini"}


def test_default_options_match_the_reference(cuda_lib):
    o = abi.Options()
    assert cuda_lib.sg_default_options(C.byref(o)) == 0
    ref = abi.default_options()
    assert bytes(o) == bytes(ref)


def test_status_strings(cuda_lib):
    assert cuda_lib.sg_status_string(0) == b"ok"
    assert cuda_lib.sg_status_string(abi.SG_ERR_CAPACITY) == b"capacity exceeded"


def test_create_without_a_device_fails_loudly(cuda_lib):
    """No CPU fallback: without a CUDA device sg_create returns an error."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    ctx = C.c_void_p()
    status = cuda_lib.sg_create(0, 4, 4, None, C.byref(ctx))
    assert status in (abi.SG_ERR_CUDA, abi.SG_ERR_INVALID)
    assert not ctx.value
    assert cuda_lib.sg_last_error(None)
