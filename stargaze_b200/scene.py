"""Scene frames in the reference's packed layout, and the f64 packer.

`Frame` mirrors `renderer::Frame` (src/renderer.rs:50-56). `pack_frame`
restates the telescope-space packing of `State::build_frame_with_vegetation`
(src/main.rs:822-1010): positions are rotated into the view frame in f64,
then split into an f32 high part and an f32 residual; stellar radiance is
`SUN_LIGHT * L / R^2` with L in solar luminosities and R in AU
(src/main.rs:71, :846). The observer frame follows `Observer::frame`
(src/camera.rs:63-120) for a non-rotating host.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

AU_M = 149_597_870_700.0  # sim::AU_KM * 1000 (src/sim.rs:13)
SOLAR_LUMINOSITY_W = 3.828e26  # nominal IAU solar luminosity
SUN_LIGHT = 2.5  # src/main.rs:71


class Frame:
    """A packed frame: Globals, bodies, ground primitives and scene time."""

    def __init__(self, globals_: abi.Globals | None = None, bodies=None, ground=None, scene_time: float = 0.0):
        self.globals = globals_ if globals_ is not None else abi.Globals()
        self.bodies: list[abi.Sphere] = list(bodies or [])
        self.ground: list[abi.Primitive] = list(ground or [])
        self.scene_time = float(scene_time)
        self._keep = None

    def view(self) -> abi.FrameView:
        """Borrowed C view; valid until the next call on this frame."""
        bodies = (abi.Sphere * max(len(self.bodies), 1))(*self.bodies)
        ground = (abi.Primitive * max(len(self.ground), 1))(*self.ground)
        g = abi.Globals.from_buffer_copy(self.globals)
        self._keep = (bodies, ground, g)
        return abi.FrameView(
            C.pointer(g),
            C.cast(bodies, C.POINTER(abi.Sphere)),
            len(self.bodies),
            C.cast(ground, C.POINTER(abi.Primitive)),
            len(self.ground),
            self.scene_time,
        )

    def copy(self) -> "Frame":
        return Frame(
            abi.Globals.from_buffer_copy(self.globals),
            [abi.Sphere.from_buffer_copy(b) for b in self.bodies],
            [abi.Primitive.from_buffer_copy(p) for p in self.ground],
            self.scene_time,
        )

    def settings(self, width: int, height: int, samples_so_far: int, count: int, max_bounces: int,
                 sampling: int, milky_way: float = 0.0, terrain_cells: int = 512) -> abi.Settings:
        """Settings exactly as `PathTracer::encode` packs them
        (src/pathtracer.rs:812-859) for a tracer of this size."""
        s = abi.Settings()
        g = abi.Globals.from_buffer_copy(self.globals)
        g.viewport[3] = g.viewport[0] / max(g.viewport[1], 1.0)
        g.viewport[0] = float(width)
        g.viewport[1] = float(height)
        g.viewport[2] = 1.0
        top = np.float32(0.0)
        for p in self.ground:
            e = np.array(p.extent[:3], dtype=np.float32)
            top = max(top, np.float32(p.center[1]) + np.sqrt(np.float32(e @ e)))
        g.ground_counts[3] = int(np.array([top], dtype=np.float32).view(np.uint32)[0])
        g.ground_counts[2] = (g.ground_counts[2] & 255) | (int(terrain_cells).bit_length() - 1) << 8
        s.g = g
        lights = [0, 0, 0, 0]
        for i, b in enumerate(self.bodies):
            if b.emissive >= 0.5:
                if lights[3] < 3:
                    lights[lights[3]] = i
                lights[3] += 1
        s.lights[:] = lights
        s.sampling[:] = [sampling & 0xFFFFFFFF, 0, 0, 0]
        s.counts[:] = [len(self.bodies), samples_so_far, count, max_bounces]
        s.background[:] = [milky_way, 1024.0, 512.0, 100.0]
        return s

    def bodies_array(self) -> C.Array:
        return (abi.Sphere * max(len(self.bodies), 1))(*self.bodies)


# ---------------------------------------------------------------------------
# Test fixtures of the reference (src/pathtracer_tests.rs:32-61,
# src/ring_tests.rs:4-10)
# ---------------------------------------------------------------------------
def frame() -> Frame:
    g = abi.Globals()
    g.cam_right[:] = [1.0, 0.0, 0.0, 0.0]
    g.cam_up[:] = [0.0, 1.0, 0.0, 0.0]
    g.cam_forward[:] = [0.0, 0.0, -1.0, 1e-7]
    g.viewport[:] = [1.0, 1.0, 1.0, 0.0]
    return Frame(g)


def body(center, radius, color, emissive: bool) -> abi.Sphere:
    b = abi.Sphere()
    b.center[:] = [float(c) for c in center]
    b.radius = float(radius)
    b.color[:] = [float(c) for c in color]
    b.emissive = 1.0 if emissive else 0.0
    return b


def ringed(center, radius, pole, tau) -> abi.Sphere:
    planet = body(center, radius, [0.0, 0.0, 0.0], False)
    planet.ring_plane[:] = [pole[0], pole[1], pole[2], 1.25]
    planet.ring_params[:] = [2.4, tau, 0.0, 0.0]
    planet.ring_color[:] = [0.8, 0.8, 0.8, 0.0]
    return planet


# ---------------------------------------------------------------------------
# f64 scene description and packing
# ---------------------------------------------------------------------------
def _unit(v) -> np.ndarray:
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


@dataclass
class Ring:
    inner_m: float
    outer_m: float
    albedo: tuple[float, float, float]
    optical_depth: float = 1.0
    banded: bool = False
    table_slot: int | None = None  # extension: tabulated tau profile
    pole: np.ndarray = field(default_factory=lambda: np.array([0.0, 0.0, 1.0]))


@dataclass
class Body:
    """A body in world coordinates (metres, watts)."""

    position_m: np.ndarray
    radius_m: float
    albedo: tuple[float, float, float] = (0.5, 0.5, 0.5)
    luminosity_w: float = 0.0
    emission: tuple[float, float, float] = (1.0, 1.0, 1.0)
    ring: Ring | None = None
    # Strength of the value-noise mottle of style-0 albedo (center_low.w,
    # pathtrace.wgsl:912-923): build_frame sets 1 on every body that is not a
    # star (src/main.rs:907); the reference's test and benchmark fixtures
    # use 0 (src/render_benchmark.rs:272-288).
    mottle: float = 1.0

    @property
    def star(self) -> bool:
        return self.luminosity_w > 0.0


@dataclass
class ViewFrame:
    """Observer frame of src/camera.rs:63-120 (world axes, AU position)."""

    position_au: np.ndarray
    forward: np.ndarray
    right: np.ndarray
    up: np.ndarray
    zenith: np.ndarray
    north: np.ndarray
    east: np.ndarray

    def world_to_view(self, v) -> np.ndarray:
        v = np.asarray(v, dtype=np.float64)
        return np.array([v @ self.right, v @ self.up, -(v @ self.forward)])


def observer_frame(host: Body, lat: float, lon: float, height_m: float, alt: float, az: float) -> ViewFrame:
    """`Observer::frame` for a host without spin (src/camera.rs:63-120)."""
    slat, clat = math.sin(lat), math.cos(lat)
    slon, clon = math.sin(lon), math.cos(lon)
    zenith = _unit([clat * clon, clat * slon, slat])
    north = np.array([-slat * clon, -slat * slon, clat])
    east = np.array([-slon, clon, 0.0])
    center_au = np.asarray(host.position_m, dtype=np.float64) / AU_M
    position = center_au + zenith * (host.radius_m / AU_M + height_m / AU_M)
    salt, calt = math.sin(alt), math.cos(alt)
    saz, caz = math.sin(az), math.cos(az)
    forward = _unit(calt * (caz * north + saz * east) + salt * zenith)
    right = _unit(caz * east - saz * north)
    up = np.cross(right, forward)
    return ViewFrame(position, forward, right, up, zenith, north, east)


def aim(host: Body, lat: float, lon: float, height_m: float, target_m) -> ViewFrame:
    """Observer frame whose forward axis points at `target_m`."""
    base = observer_frame(host, lat, lon, height_m, 0.0, 0.0)
    d = _unit(np.asarray(target_m, dtype=np.float64) / AU_M - base.position_au)
    alt = math.asin(float(np.clip(d @ base.zenith, -1.0, 1.0)))
    az = math.atan2(float(d @ base.east), float(d @ base.north))
    return observer_frame(host, lat, lon, height_m, alt, az)


def pack_frame(bodies: list[Body], view: ViewFrame, width: int, height: int, fov_y: float,
               host_index: int | None = None, height_m: float = 0.0) -> Frame:
    """`build_frame_with_vegetation` without atmosphere or landscape
    (src/main.rs:822-1010)."""
    spheres = []
    for i, b in enumerate(bodies):
        relative = np.asarray(b.position_m, dtype=np.float64) / AU_M - view.position_au
        view_center = view.world_to_view(relative)
        center = view_center.astype(np.float32)
        low = (view_center - center.astype(np.float64)).astype(np.float32)
        radius_au = b.radius_m / AU_M
        s = abi.Sphere()
        s.center[:] = [float(c) for c in center]
        s.radius = float(np.float32(radius_au))
        if b.star:
            radiance = SUN_LIGHT * (b.luminosity_w / SOLAR_LUMINOSITY_W) / radius_au**2
            s.color[:] = [float(np.float32(e * np.float32(radiance))) for e in b.emission]
            s.emissive = 1.0
        else:
            s.color[:] = list(b.albedo)
            s.emissive = 0.0
        s.center_low[:] = [float(low[0]), float(low[1]), float(low[2]), 0.0 if b.star else b.mottle]
        if b.ring is not None:
            pole = view.world_to_view(_unit(b.ring.pole))
            s.ring_plane[:] = [pole[0], pole[1], pole[2], b.ring.inner_m / b.radius_m]
            slot = 0.0 if b.ring.table_slot is None else float(b.ring.table_slot + 1)
            s.ring_params[:] = [b.ring.outer_m / b.radius_m, b.ring.optical_depth, 1.0 if b.ring.banded else 0.0, slot]
            s.ring_color[:] = [*b.ring.albedo, 0.0]
        ax = view.world_to_view([1.0, 0.0, 0.0])
        ay = view.world_to_view([0.0, 1.0, 0.0])
        s.axis_x[:] = [ax[0], ax[1], ax[2], 0.0]
        s.axis_y[:] = [ay[0], ay[1], ay[2], float(i % 4096)]
        spheres.append(s)
    g = abi.Globals()
    g.cam_right[:] = [*view.right, 0.0]
    g.cam_up[:] = [*view.up, 0.0]
    g.cam_forward[:] = [*view.forward, math.tan(fov_y * 0.5)]
    g.viewport[:] = [float(width), float(height), 1.0, 0.0]
    east = view.world_to_view(view.east)
    up = view.world_to_view(view.zenith)
    north = view.world_to_view(view.north)
    host_radius_m = bodies[host_index].radius_m if host_index is not None else 0.0
    g.ground_east[:] = [*east, height_m]
    g.ground_up[:] = [*up, host_radius_m]
    g.ground_north[:] = [*north, 0.0]
    return Frame(g, spheres)
