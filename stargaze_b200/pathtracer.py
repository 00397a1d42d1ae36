"""Python mirror of stargaze's `PathTracer` host interface (src/pathtracer.rs).

Every method is a thin call into the C-ABI library; the progressive
rendering state (history key, sample count, noise sequence) lives in the
native context, exactly where `PathTracer` keeps it in the reference.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._lib import StargazeError, check, load
from .scene import Frame


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    handle = getattr(stream, "cuda_stream", None)  # torch.cuda.Stream
    if handle is not None:
        return C.c_void_p(handle)
    raise TypeError(f"unsupported stream object {stream!r}")


def _ptr(array: np.ndarray) -> C.c_void_p:
    return C.c_void_p(array.ctypes.data)


class PathTracer:
    """`PathTracer::new(device, format, dimensions, stars, options)`
    (src/pathtracer.rs:292-302), on CUDA device `device`."""

    def __init__(self, dimensions: tuple[int, int], options: abi.Options | None = None, device: int = 0):
        self._lib = load()
        self._ctx = C.c_void_p()
        self._map_shape: tuple[int, int] | None = None
        opts = options if options is not None else abi.default_options()
        check(self._lib.sg_create(device, int(dimensions[0]), int(dimensions[1]), C.byref(opts), C.byref(self._ctx)))

    def close(self) -> None:
        if self._ctx:
            self._lib.sg_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    # -- options ----------------------------------------------------------
    @property
    def options(self) -> abi.Options:
        o = abi.Options()
        check(self._lib.sg_get_options(self._ctx, C.byref(o)), self._ctx)
        return o

    @options.setter
    def options(self, value: abi.Options) -> None:
        check(self._lib.sg_set_options(self._ctx, C.byref(value)), self._ctx)

    def update_options(self, **fields) -> None:
        o = self.options
        for k, v in fields.items():
            setattr(o, k, v)
        self.options = o

    # -- PathTracer API ---------------------------------------------------
    def resize(self, dimensions: tuple[int, int]) -> None:
        check(self._lib.sg_resize(self._ctx, int(dimensions[0]), int(dimensions[1])), self._ctx)

    def samples(self) -> int:
        s = C.c_uint32()
        check(self._lib.sg_get_samples(self._ctx, C.byref(s), None), self._ctx)
        return s.value

    def sequence(self) -> int:
        s = C.c_uint32()
        check(self._lib.sg_get_samples(self._ctx, None, C.byref(s)), self._ctx)
        return s.value

    def size(self) -> tuple[int, int]:
        w, h = C.c_uint32(), C.c_uint32()
        check(self._lib.sg_get_size(self._ctx, C.byref(w), C.byref(h)), self._ctx)
        return w.value, h.value

    def needs_redraw(self) -> bool:
        r = C.c_int()
        check(self._lib.sg_needs_redraw(self._ctx, C.byref(r)), self._ctx)
        return bool(r.value)

    def prepare_frame(self, frame: Frame) -> bool:
        fresh = C.c_int()
        view = frame.view()
        check(self._lib.sg_prepare_frame(self._ctx, C.byref(view), C.byref(fresh)), self._ctx)
        return bool(fresh.value)

    def set_fp64_sites(self, enable: bool) -> None:
        """Ring-plane and host-sphere intersections and the 5 mm offset in
        FP64 (extension; off: the reference's f32 arithmetic)."""
        check(self._lib.sg_set_fp64_sites(self._ctx, int(bool(enable))), self._ctx)

    def set_guided_ground(self, enable: bool) -> None:
        """The guided ground sampler of `PathTracer::new_with_guided_ground`
        (the reference app's default; off here as in `PathTracer::new`)."""
        check(self._lib.sg_set_guided_ground(self._ctx, int(bool(enable))), self._ctx)

    def set_ringshine(self, enable: bool) -> None:
        """Ringshine next-event estimation (pathtrace.wgsl:1248-1296), on by
        default as in the reference; off gives the integrator the
        reference's published benchmark images were rendered with. A change
        restarts the accumulation."""
        check(self._lib.sg_set_ringshine(self._ctx, int(bool(enable))), self._ctx)

    def set_checkpoints(self, every: int, max_samples: int = 0, record_bytes: int = 0) -> None:
        """Vertex checkpoints for backward() (extension): with `every` > 0
        the forward stores each path's state every `every` bounces and the
        radiance of the accumulation's first `max_samples` samples, and the
        adjoint replays segments between checkpoints instead of whole paths
        from their seeds. 0 turns it off."""
        check(self._lib.sg_set_checkpoints(self._ctx, int(every), int(max_samples), int(record_bytes)), self._ctx)

    def checkpoint_stats(self) -> dict:
        """Device bytes the checkpoints hold, records stored and records
        that did not fit."""
        b, r, d = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(self._lib.sg_get_checkpoint_stats(self._ctx, C.byref(b), C.byref(r), C.byref(d)), self._ctx)
        return {"device_bytes": b.value, "records": r.value, "dropped": d.value}

    def set_integrator(self, integrator: str, pool_paths: int = 0) -> None:
        """"wavefront" (default; stage kernels over a pool of `pool_paths`
        paths in device memory, 0 = default pool) or "megakernel" (one
        thread per pixel); both run the same per-path code and agree to a
        few ulps (extension: the reference has one compute pass)."""
        kinds = {"megakernel": abi.INTEGRATOR_MEGAKERNEL, "wavefront": abi.INTEGRATOR_WAVEFRONT}
        if integrator not in kinds:
            raise ValueError(f"unknown integrator {integrator!r}")
        check(self._lib.sg_set_integrator(self._ctx, kinds[integrator], int(pool_paths)), self._ctx)

    def integrator(self) -> dict:
        """The integrator in use, the wavefront pool of the last dispatch and
        the stage iterations it ran."""
        kind, pool, iterations = C.c_int(), C.c_uint32(), C.c_uint32()
        check(self._lib.sg_get_integrator(self._ctx, C.byref(kind), C.byref(pool), C.byref(iterations)), self._ctx)
        name = "wavefront" if kind.value == abi.INTEGRATOR_WAVEFRONT else "megakernel"
        return {"integrator": name, "pool_paths": pool.value, "iterations": iterations.value}

    STAGES = ("extend", "ring", "surface", "resolve", "gaps", "finish")

    def set_stage_timing(self, enable: bool) -> None:
        """Bracket every wavefront stage with CUDA events (measurement)."""
        check(self._lib.sg_set_stage_timing(self._ctx, int(bool(enable))), self._ctx)

    def stage_times(self) -> dict:
        """Milliseconds per wavefront stage of the last timed dispatch."""
        ms = (C.c_float * len(self.STAGES))()
        check(self._lib.sg_get_stage_times(self._ctx, ms), self._ctx)
        return dict(zip(self.STAGES, (float(v) for v in ms)))

    def set_quality(self, samples: int, bounces: int, limit: int) -> None:
        check(self._lib.sg_set_quality(self._ctx, samples, bounces, limit), self._ctx)

    def encode(self, frame: Frame, stream=None) -> None:
        view = frame.view()
        check(self._lib.sg_encode(self._ctx, C.byref(view), _stream_handle(stream)), self._ctx)

    def upload_ring_profile(self, slot: int, tau) -> None:
        t = np.ascontiguousarray(tau, dtype=np.float32)
        check(self._lib.sg_upload_ring_profile(self._ctx, slot, _ptr(t), t.size), self._ctx)

    def upload_terrain(self, data, cells: int, detail=None) -> None:
        """`Terrain::data` for a grid of `cells` cells (see terrain.py), and
        optionally the basalt elevation atlas (terrain.volcano_atlas)."""
        d = np.asarray(data, dtype=np.float32).ravel()
        if detail is not None:
            d = np.concatenate([d, np.asarray(detail, dtype=np.float32).ravel()])
        d = np.ascontiguousarray(d)
        check(self._lib.sg_upload_terrain(self._ctx, _ptr(d), d.size, cells), self._ctx)

    def upload_albedo_map(self, albedo, extent_m: float) -> None:
        """Scalar albedo map [height, width] over [-extent, extent]^2 of the
        surface frame; None removes it."""
        if albedo is None:
            check(self._lib.sg_upload_albedo_map(self._ctx, None, 0, 0, 0.0), self._ctx)
            self._map_shape = None
            return
        a = np.ascontiguousarray(albedo, dtype=np.float32)
        check(self._lib.sg_upload_albedo_map(self._ctx, _ptr(a), a.shape[1], a.shape[0], extent_m), self._ctx)
        self._map_shape = (a.shape[0], a.shape[1])

    def upload_catalogue(self, stars, cells) -> None:
        """Catalogue rows (n, 8) and cell table of stargaze_b200.sky.ray_catalogue;
        None removes the catalogue."""
        if stars is None:
            check(self._lib.sg_upload_catalogue(self._ctx, None, 0, None, 0), self._ctx)
            return
        st = np.ascontiguousarray(stars, dtype=np.float32).reshape(-1, 8)
        ce = np.ascontiguousarray(cells, dtype=np.uint32)
        check(self._lib.sg_upload_catalogue(self._ctx, _ptr(st), len(st), _ptr(ce), ce.size), self._ctx)

    def upload_milky_way(self, texels) -> None:
        """Panorama (height, width) of RGB10 texels (stargaze_b200.sky.panorama);
        None removes it."""
        if texels is None:
            check(self._lib.sg_upload_milky_way(self._ctx, None, 0, 0), self._ctx)
            return
        t = np.ascontiguousarray(texels, dtype=np.uint32)
        check(self._lib.sg_upload_milky_way(self._ctx, _ptr(t), t.shape[1], t.shape[0]), self._ctx)

    def read_pixels(self, stream=None) -> np.ndarray:
        """The accumulation as a (height*width, 4) float32 array."""
        w, h = self.size()
        out = np.zeros((w * h, 4), dtype=np.float32)
        check(self._lib.sg_read_accumulation(self._ctx, _ptr(out), 0, _stream_handle(stream)), self._ctx)
        return out

    def read_backdrop(self, stream=None) -> np.ndarray:
        w, h = self.size()
        out = np.zeros((w * h, 4), dtype=np.float32)
        check(self._lib.sg_read_backdrop(self._ctx, _ptr(out), 0, _stream_handle(stream)), self._ctx)
        return out

    def display(self, size: tuple[int, int] | None = None, linear: bool = False, stream=None) -> np.ndarray:
        """`PathTracer::display` (src/pathtracer.rs:1010-1014) into host
        memory: the exposed, ACES-mapped accumulation at `size` (default the
        trace size) as (height, width, 4) uint8 sRGB, or float32 linear."""
        w, h = size if size is not None else self.size()
        fmt = abi.DISPLAY_RGBA32F if linear else abi.DISPLAY_RGBA8_SRGB
        out = np.zeros((h, w, 4), dtype=np.float32 if linear else np.uint8)
        check(self._lib.sg_display(self._ctx, w, h, fmt, _ptr(out), 0, _stream_handle(stream)), self._ctx)
        return out

    def set_exposure_controls(self, automatic: bool, bias: float) -> None:
        """`PathTracer::set_exposure_controls` (src/pathtracer.rs:777-781)."""
        check(self._lib.sg_set_exposure_controls(self._ctx, int(bool(automatic)), float(bias)), self._ctx)

    def exposure(self, stream=None) -> float:
        """The exposure the display uses: the eased automatic value, or the
        manual one."""
        v = C.c_float()
        check(self._lib.sg_get_exposure(self._ctx, C.byref(v), _stream_handle(stream)), self._ctx)
        return v.value

    def set_accumulation(self, pixels: np.ndarray, samples: int, sequence: int) -> None:
        p = np.ascontiguousarray(pixels, dtype=np.float32)
        check(self._lib.sg_set_accumulation(self._ctx, _ptr(p), 0, samples, sequence, None), self._ctx)

    def accumulation_device_ptr(self) -> int:
        p = C.c_void_p()
        check(self._lib.sg_accumulation_device_ptr(self._ctx, C.byref(p)), self._ctx)
        return int(p.value or 0)

    def launch_count(self) -> int:
        n = C.c_uint64()
        check(self._lib.sg_launch_count(self._ctx, C.byref(n)), self._ctx)
        return n.value

    # -- probes -----------------------------------------------------------
    def closest_hit(self, frame: Frame, rays: np.ndarray) -> np.ndarray:
        """rays: structured array of abi.Ray records (see rays_array)."""
        rays = np.ascontiguousarray(rays)
        hits = np.zeros(len(rays), dtype=HIT_DTYPE)
        view = frame.view()
        check(self._lib.sg_closest_hit(self._ctx, C.byref(view), _ptr(rays), len(rays), _ptr(hits), 0, None), self._ctx)
        return hits

    def light_visibility(self, frame: Frame, rays: np.ndarray, lights) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        lights = np.ascontiguousarray(lights, dtype=np.uint32)
        out = np.zeros(len(rays), dtype=np.float32)
        view = frame.view()
        check(self._lib.sg_light_visibility(self._ctx, C.byref(view), _ptr(rays), _ptr(lights), len(rays), _ptr(out),
                                            0, None), self._ctx)
        return out

    def ring_probe(self, frame: Frame, rays: np.ndarray, body: int) -> np.ndarray:
        rays = np.ascontiguousarray(rays)
        out = np.zeros((len(rays), 4), dtype=np.float32)
        view = frame.view()
        check(self._lib.sg_ring_probe(self._ctx, C.byref(view), _ptr(rays), body, len(rays), _ptr(out), 0, None),
              self._ctx)
        return out

    def terrain_probe(self, frame: Frame, origins, directions) -> np.ndarray:
        """terrain_hit in the surface frame for each (origin, direction):
        rows of (normal xyz, distance)."""
        o = np.asarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.asarray(directions, dtype=np.float32).reshape(-1, 3)
        rays = np.ascontiguousarray(np.concatenate([o, d], axis=1))
        out = np.zeros((len(rays), 4), dtype=np.float32)
        view = frame.view()
        check(self._lib.sg_terrain_probe(self._ctx, C.byref(view), _ptr(rays), len(rays), _ptr(out), 0, None),
              self._ctx)
        return out

    def ring_energy(self, albedo: float, tau: float, mu: float, steps: int = 4096) -> float:
        e = C.c_float()
        check(self._lib.sg_ring_energy(self._ctx, albedo, tau, mu, steps, C.byref(e)), self._ctx)
        return e.value

    # -- adjoint (extension) ----------------------------------------------
    def tape(self) -> abi.Tape:
        """The replay record of the current accumulation."""
        t = abi.Tape()
        check(self._lib.sg_get_tape(self._ctx, C.byref(t)), self._ctx)
        return t

    def backward(self, frame: Frame, tape: abi.Tape, dl_dimage, stream=None) -> "Gradients":
        """Gradient of a loss with d loss / d image = `dl_dimage` ((h*w, 4) or
        (h, w, 4) float32; w channel ignored) w.r.t. the ring tables, ring
        albedos, body colours and albedo map, replaying `tape` on `frame`."""
        w, h = self.size()
        dl = np.ascontiguousarray(np.asarray(dl_dimage, dtype=np.float32).reshape(w * h, 4))
        n = len(frame.bodies)
        out = Gradients(
            ring_tau=np.zeros((abi.RING_TABLE_SLOTS, abi.RING_TABLE_MAX_BINS), dtype=np.float32),
            ring_albedo=np.zeros((n, 3), dtype=np.float32),
            body_color=np.zeros((n, 3), dtype=np.float32),
            albedo_map=np.zeros(self._map_shape, dtype=np.float32) if self._map_shape else None,
        )
        g = abi.Gradients(_ptr(out.ring_tau), _ptr(out.ring_albedo), _ptr(out.body_color),
                          _ptr(out.albedo_map) if out.albedo_map is not None else None, 0)
        view = frame.view()
        check(self._lib.sg_backward(self._ctx, C.byref(view), C.byref(tape), _ptr(dl), 0, C.byref(g),
                                    _stream_handle(stream)), self._ctx)
        out.dropped = int(g.dropped)
        return out


class Gradients:
    """d loss / d parameter blocks returned by PathTracer.backward."""

    def __init__(self, ring_tau, ring_albedo, body_color, albedo_map):
        self.ring_tau = ring_tau        # (slots, max bins)
        self.ring_albedo = ring_albedo  # (bodies, 3)
        self.body_color = body_color    # (bodies, 3)
        self.albedo_map = albedo_map    # (map height, map width) or None
        self.dropped = 0


RAY_DTYPE = np.dtype([("offset", "<f4", 3), ("direction", "<f4", 3), ("anchor", "<u4")])
HIT_DTYPE = np.dtype([("distance", "<f4"), ("index", "<u4"), ("normal", "<f4", 3)])
assert RAY_DTYPE.itemsize == C.sizeof(abi.Ray) and HIT_DTYPE.itemsize == C.sizeof(abi.Hit)


def rays_array(offsets, directions, anchors) -> np.ndarray:
    offsets = np.asarray(offsets, dtype=np.float32).reshape(-1, 3)
    directions = np.asarray(directions, dtype=np.float32).reshape(-1, 3)
    anchors = np.broadcast_to(np.asarray(anchors, dtype=np.uint32), (len(directions),))
    rays = np.zeros(len(directions), dtype=RAY_DTYPE)
    rays["offset"] = np.broadcast_to(offsets, (len(directions), 3))
    rays["direction"] = directions
    rays["anchor"] = anchors
    return rays


__all__ = ["PathTracer", "Gradients", "StargazeError", "RAY_DTYPE", "HIT_DTYPE", "rays_array"]
