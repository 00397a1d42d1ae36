"""ctypes binding of oracle/liboracle.so plus a CPU `PathTracer` stand-in.

TEST INFRASTRUCTURE ONLY (the checker). `OracleTracer` restates the host
logic of stargaze's `PathTracer` (src/pathtracer.rs:164-188 History,
:761-773 set_quality, :789-1009 encode) on top of `oracle_dispatch`, so the
reference's known-answer tests run unchanged against both the oracle and the
CUDA library.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from stargaze_b200 import abi
from stargaze_b200.pathtracer import HIT_DTYPE
from stargaze_b200.scene import Frame

ORACLE_DIR = Path(__file__).resolve().parent
LIBRARY = ORACLE_DIR / "liboracle.so"
# The same restatement with its arithmetic in f64 (-DORACLE_F64): converged
# reference images free of f32 rounding. The interface is the f32 one.
LIBRARY_F64 = ORACLE_DIR / "liboracle_f64.so"


class Tables(C.Structure):
    _fields_ = [
        ("ring_tau", C.c_void_p * abi.RING_TABLE_SLOTS),
        ("ring_bins", C.c_uint32 * abi.RING_TABLE_SLOTS),
        ("terrain", C.c_void_p),
        ("terrain_cells", C.c_uint32),
        ("terrain_detail_floats", C.c_uint32),
        ("ground", C.c_void_p),
        ("n_ground", C.c_uint32),
        ("albedo_map", C.c_void_p),
        ("map_width", C.c_uint32),
        ("map_height", C.c_uint32),
        ("map_extent", C.c_float),
        ("catalogue", C.c_void_p),
        ("catalogue_n", C.c_uint32),
        ("sky_cells", C.c_void_p),
        ("milky_way", C.c_void_p),
        ("guided_ground", C.c_uint32),
        ("ringshine_off", C.c_uint32),
    ]


class Direction(C.Structure):
    _fields_ = [
        ("ring_tau", C.c_void_p * abi.RING_TABLE_SLOTS),
        ("ring_albedo", C.c_void_p),
        ("body_color", C.c_void_p),
        ("albedo_map", C.c_void_p),
    ]


class Events(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in (
        "samples", "vertices", "sphere_tests", "sphere_hits", "ring_tests", "light_samples",
        "shadow_rays", "ring_events", "surface_events", "rng_draws", "terrain_nodes", "terrain_triangles",
        "prop_boxes", "prop_tests")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_libs: dict = {}


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return LIBRARY


def load(f64: bool = False) -> C.CDLL:
    if f64 in _libs:
        return _libs[f64]
    path = LIBRARY_F64 if f64 else LIBRARY
    if not path.exists():
        build()
    lib = C.CDLL(str(path))
    P = C.c_void_p
    S = C.POINTER(abi.Settings)
    lib.oracle_dispatch.argtypes = [S, P, C.POINTER(Tables), P, P, C.c_uint32, C.c_uint32, C.c_int, C.POINTER(Events)]
    lib.oracle_trace_sample.argtypes = [S, P, C.POINTER(Tables), C.c_uint32, C.c_uint32, C.c_uint32, P]
    lib.oracle_closest_hit.argtypes = [S, P, C.POINTER(Tables), P, C.c_uint32, P]
    lib.oracle_light_visibility.argtypes = [S, P, C.POINTER(Tables), P, P, C.c_uint32, P]
    lib.oracle_reference_visibility.argtypes = [S, P, C.POINTER(Tables), P, P, C.c_uint32, P]
    lib.oracle_ring_probe.argtypes = [S, P, C.POINTER(Tables), P, C.c_uint32, C.c_uint32, P]
    lib.oracle_ring_energy.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint32]
    lib.oracle_ring_energy.restype = C.c_float
    lib.oracle_sample_light.argtypes = [S, P, P, C.c_uint32, C.POINTER(C.c_uint32), P, C.POINTER(C.c_float)]
    lib.oracle_terrain_floats.argtypes = [C.c_uint32]
    lib.oracle_terrain_floats.restype = C.c_size_t
    lib.oracle_cache_terrain.argtypes = [P, C.c_uint32, C.c_float]
    lib.oracle_cache_terrain.restype = C.c_int
    lib.oracle_terrain_query.argtypes = [S, C.POINTER(Tables), P, P, C.c_float, C.c_int, P]
    lib.oracle_terrain_query.restype = C.c_int
    lib.oracle_sky_cache.argtypes = [S, P, C.POINTER(Tables), P]
    lib.oracle_sky_cache.restype = C.c_int
    lib.oracle_tangent.argtypes = [S, P, C.POINTER(Tables), C.POINTER(Direction), P, P, C.c_uint32, C.c_uint32,
                                   C.c_int]
    lib.oracle_tangent.restype = C.c_int
    lib.oracle_hash.argtypes = [C.c_uint32]
    lib.oracle_hash.restype = C.c_uint32
    lib.oracle_random.argtypes = [C.POINTER(C.c_uint32)]
    lib.oracle_random.restype = C.c_float
    for name in ("oracle_dispatch", "oracle_trace_sample", "oracle_closest_hit", "oracle_light_visibility",
                 "oracle_reference_visibility", "oracle_ring_probe", "oracle_sample_light"):
        getattr(lib, name).restype = C.c_int
    _libs[f64] = lib
    return lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RuntimeError(f"{what} failed with {abi.status_name(status)}")


class TableSet:
    """Scene data beyond the bodies, mirroring the CUDA context: ring
    tables, the heightfield (with its CPU-computed geometry cache) and the
    albedo map."""

    def __init__(self):
        self.tables: dict[int, np.ndarray] = {}
        self.version = 0
        self.terrain: np.ndarray | None = None
        self.terrain_cells = 0
        self.terrain_detail = 0
        self.terrain_radius: float | None = None
        self.albedo: np.ndarray | None = None
        self.map_extent = 0.0
        self._ground = None
        self.catalogue: np.ndarray | None = None
        self.sky_cells: np.ndarray | None = None
        self.milky: np.ndarray | None = None
        self.guided_ground = False
        self.ringshine = True

    def upload(self, slot: int, tau) -> None:
        self.tables[slot] = np.ascontiguousarray(tau, dtype=np.float32)
        self.version += 1

    def upload_terrain(self, data, cells: int, detail=None) -> None:
        """The reference terrain layout; `detail`, the measured elevation
        atlas of basalt ground, follows the vertex cache (volcano.rs)."""
        lib = load()
        n = lib.oracle_terrain_floats(cells)
        extra = np.zeros(0, np.float32) if detail is None else np.asarray(detail, dtype=np.float32).ravel()
        full = np.zeros(n + extra.size, dtype=np.float32)
        data = np.asarray(data, dtype=np.float32)
        full[: data.size] = data
        full[n:] = extra
        self.terrain = full
        self.terrain_cells = cells
        self.terrain_detail = int(extra.size)
        self.terrain_radius = None
        self.version += 1

    def upload_albedo_map(self, albedo, extent_m: float) -> None:
        self.albedo = None if albedo is None else np.ascontiguousarray(albedo, dtype=np.float32)
        self.map_extent = float(extent_m)
        self.version += 1

    def upload_catalogue(self, stars, cells) -> None:
        if stars is None:
            self.catalogue = self.sky_cells = None
        else:
            self.catalogue = np.ascontiguousarray(stars, dtype=np.float32).reshape(-1, 8)
            self.sky_cells = np.ascontiguousarray(cells, dtype=np.uint32)
        self.version += 1

    def upload_milky_way(self, texels) -> None:
        self.milky = None if texels is None else np.ascontiguousarray(texels, dtype=np.uint32)
        self.version += 1

    def prepare(self, frame: Frame) -> None:
        """Rebuild the terrain cache when the host radius changed (as
        src/pathtracer.rs:933-945 does on the GPU)."""
        g = frame.globals
        if self.terrain is not None and g.ground_north[3] != 0.0 and g.ground_counts[1] != 0:
            radius = float(np.float32(g.ground_up[3]))
            if self.terrain_radius != radius:
                _check(load().oracle_cache_terrain(_ptr(self.terrain), self.terrain_cells, radius), "oracle_cache_terrain")
                self.terrain_radius = radius

    def struct(self, frame: Frame | None = None) -> Tables:
        t = Tables()
        for slot, arr in self.tables.items():
            t.ring_tau[slot] = arr.ctypes.data
            t.ring_bins[slot] = arr.size
        if self.terrain is not None:
            t.terrain = self.terrain.ctypes.data
            t.terrain_cells = self.terrain_cells
            t.terrain_detail_floats = self.terrain_detail
        if frame is not None and frame.ground:
            self._ground = (abi.Primitive * len(frame.ground))(*frame.ground)
            t.ground = C.cast(self._ground, C.c_void_p)
            t.n_ground = len(frame.ground)
        if self.albedo is not None:
            t.albedo_map = self.albedo.ctypes.data
            t.map_width = self.albedo.shape[1]
            t.map_height = self.albedo.shape[0]
            t.map_extent = self.map_extent
        if self.catalogue is not None:
            t.catalogue = self.catalogue.ctypes.data
            t.catalogue_n = len(self.catalogue)
            t.sky_cells = self.sky_cells.ctypes.data
        if self.milky is not None:
            t.milky_way = self.milky.ctypes.data
        t.guided_ground = 1 if self.guided_ground else 0
        t.ringshine_off = 0 if self.ringshine else 1
        return t


def frame_bytes(frame: Frame) -> bytes:
    out = bytes(frame.globals)
    out += b"".join(bytes(b) for b in frame.bodies)
    out += b"".join(bytes(p) for p in frame.ground)
    out += np.float64(frame.scene_time).tobytes()
    return out


class OracleTracer:
    """CPU restatement of the `PathTracer` host contract on the oracle."""

    def __init__(self, dimensions, options: abi.Options | None = None, threads: int = 0, f64: bool = False):
        self.lib = load(f64)
        self.width, self.height = int(dimensions[0]), int(dimensions[1])
        self.opts = abi.Options.from_buffer_copy(options if options is not None else abi.default_options())
        self.threads = threads
        self.key = None
        self.samples_ = 0
        self.sequence_ = 0
        self.idle = 0
        self.tables = TableSet()
        self.acc = np.zeros((self.width * self.height, 4), dtype=np.float32)
        self.backdrop = np.zeros_like(self.acc)
        self.events = Events()

    # options mirror
    @property
    def options(self) -> abi.Options:
        return abi.Options.from_buffer_copy(self.opts)

    @options.setter
    def options(self, value: abi.Options) -> None:
        self.opts = abi.Options.from_buffer_copy(value)

    def update_options(self, **fields) -> None:
        for k, v in fields.items():
            setattr(self.opts, k, v)

    def resize(self, dimensions) -> None:
        w, h = int(dimensions[0]), int(dimensions[1])
        if (w, h) == (self.width, self.height):
            return
        self.width, self.height = w, h
        self.acc = np.zeros((w * h, 4), dtype=np.float32)
        self.backdrop = np.zeros_like(self.acc)
        self.key = None
        self.samples_ = 0
        self.idle = 0

    def samples(self) -> int:
        return self.samples_

    def sequence(self) -> int:
        return self.sequence_

    def size(self):
        return self.width, self.height

    def needs_redraw(self) -> bool:
        return self.samples_ < self.opts.sample_limit or (bool(self.opts.auto_exposure) and self.idle < 60)

    def _update_history(self, frame: Frame) -> None:
        key = frame_bytes(frame) + np.uint32(self.opts.max_bounces).tobytes() + \
            np.float32(self.opts.milky_way).tobytes() + np.uint64(self.tables.version).tobytes()
        if key != self.key:
            self.key = key
            self.samples_ = 0

    def prepare_frame(self, frame: Frame) -> bool:
        self._update_history(frame)
        return self.samples_ == 0

    def set_quality(self, samples: int, bounces: int, limit: int) -> None:
        bounces = min(max(bounces, 1), 64)
        if self.opts.max_bounces != bounces:
            self.key = None
            self.samples_ = 0
            self.idle = 0
        self.opts.samples_per_frame = min(max(samples, 1), 64)
        self.opts.max_bounces = bounces
        self.opts.sample_limit = min(max(limit, 1), abi.MAX_SAMPLES)

    def upload_ring_profile(self, slot: int, tau) -> None:
        self.tables.upload(slot, tau)

    def upload_terrain(self, data, cells: int, detail=None) -> None:
        self.tables.upload_terrain(data, cells, detail)

    def upload_albedo_map(self, albedo, extent_m: float) -> None:
        self.tables.upload_albedo_map(albedo, extent_m)

    def settings_for(self, frame: Frame, count: int) -> abi.Settings:
        s = frame.settings(self.width, self.height, self.samples_, count, self.opts.max_bounces,
                           self.opts.noise_seed + self.sequence_, self.opts.milky_way,
                           terrain_cells=self.tables.terrain_cells or 512)
        if self.tables.milky is not None:
            s.background[1] = float(self.tables.milky.shape[1])
            s.background[2] = float(self.tables.milky.shape[0])
        return s

    def upload_catalogue(self, stars, cells) -> None:
        self.tables.upload_catalogue(stars, cells)

    def upload_milky_way(self, texels) -> None:
        self.tables.upload_milky_way(texels)

    def set_guided_ground(self, enable: bool) -> None:
        """The guided ground sampler (src/guided_ground.rs:14-79); like a
        new tracer, a change restarts the accumulation."""
        if bool(enable) != self.tables.guided_ground:
            self.tables.guided_ground = bool(enable)
            self.tables.version += 1

    def set_ringshine(self, enable: bool) -> None:
        """Ringshine next-event estimation (pathtrace.wgsl:1248-1296), on by
        default; a change restarts the accumulation."""
        if bool(enable) != self.tables.ringshine:
            self.tables.ringshine = bool(enable)
            self.tables.version += 1

    def encode(self, frame: Frame, stream=None, rows=None) -> None:
        if len(frame.bodies) > abi.BODY_CAPACITY:
            raise RuntimeError("too many scene bodies")
        self._update_history(frame)
        count = min(self.opts.samples_per_frame, abi.MAX_BATCH_SAMPLES, max(self.opts.sample_limit - self.samples_, 0))
        if count > 0:
            s = self.settings_for(frame, count)
            bodies = frame.bodies_array()
            self.tables.prepare(frame)
            t = self.tables.struct(frame)
            y0, y1 = rows if rows is not None else (0, self.height)
            _check(self.lib.oracle_dispatch(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(self.acc),
                                            _ptr(self.backdrop), y0, y1, self.threads, C.byref(self.events)),
                   "oracle_dispatch")
        self.samples_ += count
        self.sequence_ = (self.sequence_ + count) & 0xFFFFFFFF
        self.idle = 0 if count > 0 else self.idle + 1

    def read_pixels(self) -> np.ndarray:
        return self.acc.copy()

    def read_backdrop(self) -> np.ndarray:
        return self.backdrop.copy()

    # probes -------------------------------------------------------------
    def _probe_args(self, frame: Frame):
        s = self.settings_for(frame, 0)
        self.tables.prepare(frame)
        return s, frame.bodies_array(), self.tables.struct(frame)

    def terrain_probe(self, frame: Frame, origins, directions) -> np.ndarray:
        """Mirror of PathTracer.terrain_probe: terrain_hit per ray."""
        o = np.asarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.asarray(directions, dtype=np.float32).reshape(-1, 3)
        return np.array([self.terrain_query(frame, o[k], d[k]) for k in range(len(o))], dtype=np.float32)

    def terrain_query(self, frame: Frame, o, d, limit: float = 1.0e29, occlusion: bool = False) -> np.ndarray:
        """terrain_query in the surface frame: (normal xyz, distance)."""
        s, _bodies, t = self._probe_args(frame)
        o = np.ascontiguousarray(o, dtype=np.float32)
        d = np.ascontiguousarray(d, dtype=np.float32)
        out = np.zeros(4, dtype=np.float32)
        _check(self.lib.oracle_terrain_query(C.byref(s), C.byref(t), _ptr(o), _ptr(d), limit, int(occlusion),
                                             _ptr(out)), "oracle_terrain_query")
        return out

    def sky_cache(self, frame: Frame) -> np.ndarray:
        """The surface sky cache of `frame` (terrain.wgsl:286-302): (8, 16, 4)
        texels by elevation row and azimuth."""
        s, bodies, t = self._probe_args(frame)
        out = np.zeros((8, 16, 4), dtype=np.float32)
        _check(self.lib.oracle_sky_cache(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(out)),
               "oracle_sky_cache")
        return out

    def closest_hit(self, frame: Frame, rays: np.ndarray) -> np.ndarray:
        s, bodies, t = self._probe_args(frame)
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        _check(self.lib.oracle_closest_hit(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(rays), len(rays),
                                           _ptr(hits)), "oracle_closest_hit")
        return hits

    def light_visibility(self, frame: Frame, rays: np.ndarray, lights) -> np.ndarray:
        s, bodies, t = self._probe_args(frame)
        rays = np.ascontiguousarray(rays)
        lights = np.ascontiguousarray(lights, dtype=np.uint32)
        out = np.zeros(len(rays), dtype=np.float32)
        _check(self.lib.oracle_light_visibility(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(rays),
                                                _ptr(lights), len(rays), _ptr(out)), "oracle_light_visibility")
        return out

    def reference_visibility(self, frame: Frame, rays: np.ndarray, lights) -> np.ndarray:
        s, bodies, t = self._probe_args(frame)
        rays = np.ascontiguousarray(rays)
        lights = np.ascontiguousarray(lights, dtype=np.uint32)
        out = np.zeros(len(rays), dtype=np.float32)
        _check(self.lib.oracle_reference_visibility(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(rays),
                                                    _ptr(lights), len(rays), _ptr(out)), "oracle_reference_visibility")
        return out

    def ring_probe(self, frame: Frame, rays: np.ndarray, body: int) -> np.ndarray:
        s, bodies, t = self._probe_args(frame)
        rays = np.ascontiguousarray(rays)
        out = np.zeros((len(rays), 4), dtype=np.float32)
        _check(self.lib.oracle_ring_probe(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), _ptr(rays), body,
                                          len(rays), _ptr(out)), "oracle_ring_probe")
        return out

    def ring_energy(self, albedo: float, tau: float, mu: float, steps: int = 4096) -> float:
        return float(self.lib.oracle_ring_energy(albedo, tau, mu, steps))

    def tangent(self, frame: Frame, first: int, count: int, ring_tau=None, ring_albedo=None, body_color=None,
                albedo_map=None, rows=None):
        """Forward-mode derivative of the samples with noise keys
        [first, first + count) along a parameter direction: ring_tau maps a
        table slot to per-bin tangents, ring_albedo / body_color are
        (bodies, 3), albedo_map matches the uploaded map. Returns the
        per-pixel sums (primal, tangent), each (height*width, 4)."""
        n = len(frame.bodies)
        keep = []

        def arr(a, shape=None):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32)
            if shape is not None:
                a = a.reshape(shape)
            keep.append(a)
            return a.ctypes.data

        d = Direction()
        for slot, t in (ring_tau or {}).items():
            d.ring_tau[slot] = arr(t)
        d.ring_albedo = arr(ring_albedo, (n, 3))
        d.body_color = arr(body_color, (n, 3))
        d.albedo_map = arr(albedo_map)
        primal = np.zeros((self.width * self.height, 4), dtype=np.float32)
        tangent = np.zeros_like(primal)
        bodies = frame.bodies_array()
        self.tables.prepare(frame)
        t = self.tables.struct(frame)
        y0, y1 = rows if rows is not None else (0, self.height)
        done = 0
        while done < count:
            batch = min(abi.MAX_BATCH_SAMPLES, count - done)
            s = self.settings_for(frame, batch)
            s.sampling[0] = (first + done) & 0xFFFFFFFF
            _check(self.lib.oracle_tangent(C.byref(s), C.cast(bodies, C.c_void_p), C.byref(t), C.byref(d),
                                           _ptr(primal), _ptr(tangent), y0, y1, self.threads), "oracle_tangent")
            done += batch
        return primal, tangent

    def trace_sample(self, frame: Frame, x: int, y: int, s: int) -> np.ndarray:
        st, bodies, t = self._probe_args(frame)
        st.counts[2] = 1
        out = np.zeros(4, dtype=np.float32)
        _check(self.lib.oracle_trace_sample(C.byref(st), C.cast(bodies, C.c_void_p), C.byref(t), x, y, s, _ptr(out)),
               "oracle_trace_sample")
        return out


def oracle_hash(value: int) -> int:
    return int(load().oracle_hash(value & 0xFFFFFFFF))


def oracle_random(state: int) -> tuple[float, int]:
    st = C.c_uint32(state & 0xFFFFFFFF)
    value = load().oracle_random(C.byref(st))
    return float(value), st.value
