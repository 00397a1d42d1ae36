"""Loader for the in-tree C-ABI library `libstargaze_b200.so`.

There is no CPU fallback: if the CUDA library is missing or cannot be
loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import abi

LIBRARY_PATH = Path(__file__).resolve().parent / "libstargaze_b200.so"

# Every entry point declared in include/stargaze_b200.h, with ctypes types.
_P = C.c_void_p
_SIGNATURES = {
    "sg_default_options": (C.c_int, [C.POINTER(abi.Options)]),
    "sg_create": (C.c_int, [C.c_int, C.c_uint32, C.c_uint32, C.POINTER(abi.Options), C.POINTER(_P)]),
    "sg_destroy": (C.c_int, [_P]),
    "sg_resize": (C.c_int, [_P, C.c_uint32, C.c_uint32]),
    "sg_prepare_frame": (C.c_int, [_P, C.POINTER(abi.FrameView), C.POINTER(C.c_int)]),
    "sg_set_quality": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint32]),
    "sg_set_options": (C.c_int, [_P, C.POINTER(abi.Options)]),
    "sg_get_options": (C.c_int, [_P, C.POINTER(abi.Options)]),
    "sg_encode": (C.c_int, [_P, C.POINTER(abi.FrameView), _P]),
    "sg_get_samples": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "sg_needs_redraw": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "sg_get_size": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "sg_read_accumulation": (C.c_int, [_P, _P, C.c_int, _P]),
    "sg_read_backdrop": (C.c_int, [_P, _P, C.c_int, _P]),
    "sg_set_accumulation": (C.c_int, [_P, _P, C.c_int, C.c_uint32, C.c_uint32, _P]),
    "sg_accumulation_device_ptr": (C.c_int, [_P, C.POINTER(_P)]),
    "sg_upload_ring_profile": (C.c_int, [_P, C.c_uint32, _P, C.c_uint32]),
    "sg_upload_terrain": (C.c_int, [_P, _P, C.c_size_t, C.c_uint32]),
    "sg_upload_albedo_map": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32, C.c_float]),
    "sg_closest_hit": (C.c_int, [_P, C.POINTER(abi.FrameView), _P, C.c_uint32, _P, C.c_int, _P]),
    "sg_light_visibility": (C.c_int, [_P, C.POINTER(abi.FrameView), _P, _P, C.c_uint32, _P, C.c_int, _P]),
    "sg_ring_probe": (C.c_int, [_P, C.POINTER(abi.FrameView), _P, C.c_uint32, C.c_uint32, _P, C.c_int, _P]),
    "sg_ring_energy": (C.c_int, [_P, C.c_float, C.c_float, C.c_float, C.c_uint32, C.POINTER(C.c_float)]),
    "sg_terrain_probe": (C.c_int, [_P, C.POINTER(abi.FrameView), _P, C.c_uint32, _P, C.c_int, _P]),
    "sg_last_error": (C.c_char_p, [_P]),
    "sg_status_string": (C.c_char_p, [C.c_int]),
    "sg_launch_count": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "sg_encode_counted": (C.c_int, [_P, C.POINTER(abi.FrameView), _P, C.POINTER(C.c_uint64)]),
    "sg_measure_fp32_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "sg_closest_hit_noalloc": (C.c_int, [C.c_int, C.POINTER(abi.FrameView), _P, C.c_uint32, _P, _P]),
    "sg_set_fp64_sites": (C.c_int, [_P, C.c_int]),
    "sg_set_guided_ground": (C.c_int, [_P, C.c_int]),
    "sg_set_ringshine": (C.c_int, [_P, C.c_int]),
    "sg_set_checkpoints": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_uint64]),
    "sg_get_checkpoint_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "sg_set_integrator": (C.c_int, [_P, C.c_int, C.c_uint32]),
    "sg_get_integrator": (C.c_int, [_P, C.POINTER(C.c_int), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "sg_set_stage_timing": (C.c_int, [_P, C.c_int]),
    "sg_display": (C.c_int, [_P, C.c_uint32, C.c_uint32, C.c_int, _P, C.c_int, _P]),
    "sg_upload_catalogue": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32]),
    "sg_upload_milky_way": (C.c_int, [_P, _P, C.c_uint32, C.c_uint32]),
    "sg_get_exposure": (C.c_int, [_P, C.POINTER(C.c_float), _P]),
    "sg_set_exposure_controls": (C.c_int, [_P, C.c_int, C.c_float]),
    "sg_get_stage_times": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "sg_get_tape": (C.c_int, [_P, C.POINTER(abi.Tape)]),
    "sg_backward": (C.c_int, [_P, C.POINTER(abi.FrameView), C.POINTER(abi.Tape), _P, C.c_int,
                              C.POINTER(abi.Gradients), _P]),
}

_lib: C.CDLL | None = None


class StargazeError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.status_name(status)}: {message}")
        self.status = status


def exported_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def load(path: Path | None = None) -> C.CDLL:
    """Load (once) and type the library. Raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(path) if path else LIBRARY_PATH
    if not path.exists():
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()')"
        )
    lib = C.CDLL(str(path))
    for name, (restype, argtypes) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != abi.SG_OK:
        lib = load()
        message = lib.sg_last_error(ctx)
        raise StargazeError(status, message.decode() if message else "")
