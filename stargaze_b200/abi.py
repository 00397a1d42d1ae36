"""ctypes mirror of include/stargaze_b200.h.

The structures are byte-identical to the reference's `bytemuck` structs:
`Globals` (src/renderer.rs:15-31, 176 B), `Settings` (src/pathtracer.rs:46-52,
240 B), `Sphere` (src/renderer.rs:35-48, 160 B) and `ground::Primitive`
(src/shaders/ground.wgsl:3-7, 48 B). The reference checks the same spans
against the WGSL structs in `validate_shaders_and_buffer_layouts`
(src/pathtracer_tests.rs:63-97).
"""
from __future__ import annotations

import ctypes as C

F4 = C.c_float * 4
F3 = C.c_float * 3
U4 = C.c_uint32 * 4

SG_OK = 0
SG_ERR_INVALID = -1
SG_ERR_CAPACITY = -2
SG_ERR_CUDA = -3
SG_ERR_OOM = -4
SG_ERR_STATE = -5
SG_ERR_TIMEOUT = -6

BODY_CAPACITY = 256
MAX_BATCH_SAMPLES = 64
GROUND_CAPACITY = 256
MAX_SAMPLES = 16_777_216
RING_TABLE_SLOTS = 8
RING_TABLE_MAX_BINS = 4096
MISS = 0xFFFFFFFF
LOCAL_BASE = 0x80000000
TERRAIN_ID = 0x80100000


class Globals(C.Structure):
    _fields_ = [
        ("cam_right", F4),
        ("cam_up", F4),
        ("cam_forward", F4),
        ("viewport", F4),
        ("atmo_center", F4),
        ("atmo_rayleigh", F4),
        ("atmo_params", F4),
        ("ground_east", F4),
        ("ground_up", F4),
        ("ground_north", F4),
        ("ground_counts", U4),
    ]


class Settings(C.Structure):
    _fields_ = [
        ("g", Globals),
        ("counts", U4),
        ("sampling", U4),
        ("background", F4),
        ("lights", U4),
    ]


class Sphere(C.Structure):
    _fields_ = [
        ("center", F3),
        ("radius", C.c_float),
        ("color", F3),
        ("emissive", C.c_float),
        ("center_low", F4),
        ("ring_plane", F4),
        ("ring_params", F4),
        ("ring_color", F4),
        ("axis_x", F4),
        ("axis_y", F4),
        ("surface_color", F4),
        ("surface_params", F4),
    ]


class Primitive(C.Structure):
    _fields_ = [("center", F4), ("extent", F4), ("albedo", F4)]


class Options(C.Structure):
    _fields_ = [
        ("noise_seed", C.c_uint32),
        ("samples_per_frame", C.c_uint32),
        ("max_bounces", C.c_uint32),
        ("sample_limit", C.c_uint32),
        ("exposure", C.c_float),
        ("auto_exposure", C.c_int32),
        ("ev_bias", C.c_float),
        ("auto_key", C.c_float),
        ("auto_percentile", C.c_float),
        ("milky_way", C.c_float),
    ]


class FrameView(C.Structure):
    """Borrowed view of a `renderer::Frame` (src/renderer.rs:50-56)."""

    _fields_ = [
        ("globals", C.POINTER(Globals)),
        ("bodies", C.POINTER(Sphere)),
        ("n_bodies", C.c_uint32),
        ("ground", C.POINTER(Primitive)),
        ("n_ground", C.c_uint32),
        ("scene_time", C.c_double),
    ]


class Ray(C.Structure):
    _fields_ = [("offset", F3), ("direction", F3), ("anchor", C.c_uint32)]


class Hit(C.Structure):
    _fields_ = [("distance", C.c_float), ("index", C.c_uint32), ("normal", F3)]


NOALLOC_MAX_RAYS = 65536
DISPLAY_RGBA8_SRGB = 0
DISPLAY_RGBA32F = 1
INTEGRATOR_MEGAKERNEL = 0
INTEGRATOR_WAVEFRONT = 1
WAVE_MAX_POOL = 1 << 26
NOALLOC_SCRATCH_BYTES = 4 << 20
TAPE_RANGES = 16


class Tape(C.Structure):
    """Replay record of an accumulation (extension: the adjoint's saved state)."""

    _fields_ = [
        ("width", C.c_uint32),
        ("height", C.c_uint32),
        ("samples", C.c_uint32),
        ("n_ranges", C.c_uint32),
        ("first", C.c_uint32 * TAPE_RANGES),
        ("count", C.c_uint32 * TAPE_RANGES),
        ("history_hash", C.c_uint64),
    ]


class Gradients(C.Structure):
    _fields_ = [
        ("ring_tau", C.c_void_p),
        ("ring_albedo", C.c_void_p),
        ("body_color", C.c_void_p),
        ("albedo_map", C.c_void_p),
        ("dropped", C.c_uint64),
    ]


LAYOUT_SIZES = {
    "Globals": (Globals, 176),
    "Settings": (Settings, 240),
    "Sphere": (Sphere, 160),
    "Primitive": (Primitive, 48),
    "Ray": (Ray, 28),
    "Hit": (Hit, 20),
    "Tape": (Tape, 152),
    "Gradients": (Gradients, 40),
}


def default_options() -> Options:
    """`Options::default()` (src/pathtracer.rs:95-111)."""
    return Options(
        noise_seed=0,
        samples_per_frame=1,
        max_bounces=8,
        sample_limit=MAX_SAMPLES,
        exposure=1.0,
        auto_exposure=0,
        ev_bias=0.0,
        auto_key=0.25,
        auto_percentile=0.9,
        milky_way=4.0e-4,
    )


def status_name(code: int) -> str:
    return {
        SG_OK: "SG_OK",
        SG_ERR_INVALID: "SG_ERR_INVALID",
        SG_ERR_CAPACITY: "SG_ERR_CAPACITY",
        SG_ERR_CUDA: "SG_ERR_CUDA",
        SG_ERR_OOM: "SG_ERR_OOM",
        SG_ERR_STATE: "SG_ERR_STATE",
        SG_ERR_TIMEOUT: "SG_ERR_TIMEOUT",
    }.get(code, f"status {code}")
