"""Seeded synthetic workloads in the reference's packed layout.

No reference scene files are involved: each workload is synthesised in f64
from its physical description and packed like `build_frame` does
(src/main.rs:822-1010). Random choices use SplitMix64 with the stated seed.

* `spheres_256`: 256x256, 64 spp, max depth 6. A star (R 7.0e8 m, L 3.8e26 W)
  1.5e11 m along +x; a Lambertian host (R 6.4e6 m, albedo 0.3) at the origin;
  a moon (R 1.74e6 m, albedo 0.12) 3.84e8 m away at 100 degrees longitude.
  The camera stands 2 m above the host at 35 N, 30 E (mid-afternoon), 60
  degree vertical field of view, aimed at the moon (16 degrees up), so the
  lower quarter of the frame is sunlit ground.
* `rings_1080p`: 1920x1080, 256 spp. A gas giant (R 5.8e7 m, albedo 0.5) with
  an equatorial ring from 7.4e7 m to 1.37e8 m whose optical depth comes from
  a 512-bin table (C/B/A-like bands, tau in [0, 2], seeded gap bins at 0),
  single-scattering albedo 0.5. Two stars (9e8 m / 5e26 W and 5e8 m /
  1e26 W) in a 3e11 m circular binary whose barycentre lies 1.5e12 m from
  the planet. A moon (R 1.5e6 m) orbits 2e8 m out, 8 degrees off the
  planet-to-nearer-star line, so its shadow (a partial eclipse of that star)
  falls on the planet's disc. The camera stands 2 m above the moon on its
  planet-facing side, 80 degree field of view, aimed at the planet, which
  rides 30 degrees above the moon's horizon.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import abi
from .scene import AU_M, Body, Frame, Ring, aim, pack_frame


def splitmix64(seed: int):
    """SplitMix64 generator (Steele, Lea & Flood 2014)."""
    state = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield z ^ (z >> 31)


def uniform01(gen, n: int) -> np.ndarray:
    return np.array([(next(gen) >> 11) * (1.0 / 9007199254740992.0) for _ in range(n)])


@dataclass
class Workload:
    name: str
    frame: Frame
    width: int
    height: int
    spp: int
    max_bounces: int
    ring_tables: dict[int, np.ndarray]
    description: str
    landscape: object = None  # LandscapeData for scenes with terrain

    @property
    def samples(self) -> int:
        return self.width * self.height * self.spp


def ring_tau_profile(bins: int = 512, seed: int = 0, gaps: int = 12) -> np.ndarray:
    """C/B/A-like optical-depth bands on the normalised ring radius.

    Band edges follow the fractions of the reference's banded profile
    (src/shaders/rings.wgsl:62-71): C ring below 0.2792, B ring to 0.6910,
    the Cassini division to 0.7649, then the A ring. `gaps` bins chosen with
    SplitMix64(seed) are emptied (tau = 0). Values are clamped to [0, 2].
    """
    x = (np.arange(bins, dtype=np.float64) + 0.5) / bins
    broad = 0.5 + 0.5 * np.sin(43.0 * x + 1.8 * np.sin(17.0 * x))
    tau = np.where(x < 0.2792, 0.08 + 0.06 * broad, 0.0)
    tau = np.where((x >= 0.2792) & (x < 0.6910), 1.1 + 0.8 * broad, tau)
    tau = np.where((x >= 0.6910) & (x < 0.7649), 0.04, tau)
    tau = np.where(x >= 0.7649, 0.45 + 0.3 * broad, tau)
    gen = splitmix64(seed)
    picks = set()
    while len(picks) < gaps:
        picks.add(int(next(gen) % bins))
    for k in sorted(picks):
        tau[k] = 0.0
    return np.clip(tau, 0.0, 2.0).astype(np.float32)


# The benchmark scenes have Lambertian bodies of constant albedo: mottle 0,
# as the reference's own test and benchmark fixtures set it
# (src/render_benchmark.rs:272-288); with_mottle() turns it on as the app's
# build_frame does.


def with_mottle(frame, strength: float = 1.0):
    """center_low.w = `strength` on every body that is not a star
    (src/main.rs:907): the style-0 albedo's value-noise mottle."""
    for b in frame.bodies:
        if b.emissive < 0.5:
            b.center_low[3] = strength
    return frame


def spheres_256(width: int = 256, height: int = 256, spp: int = 64) -> Workload:
    star = Body(np.array([1.5e11, 0.0, 0.0]), 7.0e8, luminosity_w=3.8e26)
    host = Body(np.zeros(3), 6.4e6, albedo=(0.3, 0.3, 0.3), mottle=0.0)
    moon_dir = np.array([math.cos(math.radians(100.0)), math.sin(math.radians(100.0)), 0.0])
    moon = Body(3.84e8 * moon_dir, 1.74e6, albedo=(0.12, 0.12, 0.12), mottle=0.0)
    bodies = [star, host, moon]
    view = aim(host, math.radians(35.0), math.radians(30.0), 2.0, moon.position_m)
    frame = pack_frame(bodies, view, width, height, math.radians(60.0), host_index=1, height_m=2.0)
    return Workload("spheres_256", frame, width, height, spp, 6, {}, "3 spheres, star NEE, depth 6")


def rings_1080p(width: int = 1920, height: int = 1080, spp: int = 256, max_bounces: int = 6) -> Workload:
    planet_pos = np.zeros(3)
    barycentre = np.array([1.5e12, 0.0, 0.0])
    phase = math.radians(60.0)
    axis = np.array([math.cos(phase), math.sin(phase), 0.25])
    axis /= np.linalg.norm(axis)
    star_a = Body(barycentre - 1.0e11 * axis, 9.0e8, luminosity_w=5.0e26)
    star_b = Body(barycentre + 2.0e11 * axis, 5.0e8, luminosity_w=1.0e26)
    nearer = star_a if np.linalg.norm(star_a.position_m) < np.linalg.norm(star_b.position_m) else star_b
    to_star = nearer.position_m / np.linalg.norm(nearer.position_m)
    side = np.cross(to_star, [0.0, 0.0, 1.0])
    side /= np.linalg.norm(side)
    off = math.radians(8.0)
    moon_dir = math.cos(off) * to_star + math.sin(off) * side
    moon = Body(planet_pos + 2.0e8 * moon_dir, 1.5e6, albedo=(0.12, 0.12, 0.12), mottle=0.0)
    pole = np.array([0.3, 0.2, 0.93])
    ring = Ring(7.4e7, 1.37e8, (0.5, 0.5, 0.5), optical_depth=1.0, table_slot=0, pole=pole / np.linalg.norm(pole))
    planet = Body(planet_pos, 5.8e7, albedo=(0.5, 0.5, 0.5), ring=ring, mottle=0.0)
    bodies = [star_a, star_b, planet, moon]
    # Camera zenith: rotate the moon-to-planet direction 60 degrees towards
    # the ring pole so the planet stands 30 degrees above the horizon.
    to_planet = -moon_dir
    tilt = np.cross(to_planet, np.cross(pole, to_planet))
    tilt /= np.linalg.norm(tilt)
    zenith = math.cos(math.radians(60.0)) * to_planet + math.sin(math.radians(60.0)) * tilt
    lat = math.asin(zenith[2])
    lon = math.atan2(zenith[1], zenith[0])
    view = aim(moon, lat, lon, 2.0, planet_pos)
    frame = pack_frame(bodies, view, width, height, math.radians(80.0), host_index=3, height_m=2.0)
    tables = {0: ring_tau_profile(512, seed=0)}
    return Workload("rings_1080p", frame, width, height, spp, max_bounces, tables,
                    "ringed giant, 512-bin tau table, binary star, moon eclipse")


@dataclass
class LandscapeData:
    heights: np.ndarray
    terrain: np.ndarray  # reference layout (heights, bounds)
    cells: int
    albedo_map: np.ndarray | None = None
    map_extent: float = 0.0
    detail: np.ndarray | None = None  # basalt elevation atlas (terrain.volcano_atlas)


def terrain_1080p(width: int = 1920, height: int = 1080, spp: int = 128, cells: int = 4096,
                  rocks: int = 2000, foliage: int = 5000, max_bounces: int = 6, seed: int = 0,
                  prop_range: tuple[float, float] = (25.0, 2000.0)):
    """Terrain and precision scene: a 6.4e6 m host carrying a `cells`^2
    seeded fBm heightfield (8 octaves, 300 m amplitude) under the min/max
    quadtree, lifted so its lowest vertex is 0.5 m above the host sphere,
    `rocks` faceted rocks and boxes and `foliage` ellipsoids in a
    group-marker BVH between `prop_range` metres of the observer, one star 20
    degrees above the horizon; the camera 2 m above the terrain, looking 4
    degrees down, 70 degree field of view. Returns (Workload, LandscapeData)."""
    from . import terrain as T

    heights = T.fbm_heights(cells, seed=seed)
    heights = (heights - heights.min() + 0.5).astype(np.float32)
    centre = (cells + 1) * (cells // 2) + cells // 2
    observer_m = float(heights[centre]) + 2.0  # 2 m above the terrain
    terrain = T.pack_terrain(heights, cells)

    R = 6.4e6
    host = Body(np.zeros(3), R, albedo=(0.3, 0.3, 0.3), mottle=0.0)
    lat, lon = math.radians(35.0), math.radians(30.0)
    base = aim(host, lat, lon, observer_m, np.array([1.0e9, 0.0, 0.0]))
    # Star: azimuth 140 degrees (south-east), 20 degrees above the horizon.
    alt, az = math.radians(20.0), math.radians(140.0)
    sdir = math.cos(alt) * (math.cos(az) * base.north + math.sin(az) * base.east) + math.sin(alt) * base.zenith
    star = Body(base.position_au * AU_M + 1.5e11 * sdir, 7.0e8, luminosity_w=3.8e26)
    # View: azimuth 100 degrees, 4 degrees down.
    valt, vaz = math.radians(-4.0), math.radians(100.0)
    target = base.position_au * AU_M + 1.0e4 * (math.cos(valt) * (math.cos(vaz) * base.north +
                                                               math.sin(vaz) * base.east) + math.sin(valt) * base.zenith)
    view = aim(host, lat, lon, observer_m, target)
    bodies = [star, host]
    frame = pack_frame(bodies, view, width, height, math.radians(70.0), host_index=1, height_m=observer_m)
    frame.globals.ground_north[3] = 2.0  # host index + 1: the landscape is on

    gen = splitmix64(seed + 11)
    near, far = prop_range
    # View direction in the surface frame (x east, z north).
    fwd = np.array([math.sin(vaz), 0.0, math.cos(vaz)])
    side = np.array([fwd[2], 0.0, -fwd[0]])
    props = []
    for k in range(rocks + foliage):
        u = uniform01(gen, 4)
        dist = near + (far - near) * math.sqrt(u[0])  # uniform over the ground area
        lateral = (u[1] - 0.5) * 1.8 * dist
        x, z = fwd[0] * dist + side[0] * lateral, fwd[2] * dist + side[2] * lateral
        ground = T.height_at(heights, cells, x, z, R)
        if k < rocks:
            e = np.array([0.3 + 1.5 * u[2], 0.25 + 1.0 * u[3], 0.3 + 1.5 * u[2] * 0.8])
            if k % 3 == 0:
                kind, yaw = 0.0, 0.0  # plain box
            elif k % 3 == 1:
                kind, yaw = 2.0, (u[3] - 0.5) * 0.6  # faceted rock, leaning
            else:
                angles = [int(255 * v) for v in uniform01(gen, 3)]
                kind, yaw = 2.25, float(angles[0] | (angles[1] << 8) | (angles[2] << 16))
            tint = (0.28 + 0.1 * u[3], 0.27 + 0.08 * u[2], 0.25 + 0.06 * u[1])
            props.append(T.primitive([x, ground + 0.6 * e[1], z], kind, e, yaw, tint, 1.0))
        else:
            e = np.array([0.6 + 1.4 * u[2], 1.0 + 3.0 * u[3], 0.6 + 1.4 * u[2]])
            tint = (0.05 + 0.05 * u[3], 0.12 + 0.1 * u[2], 0.04 + 0.03 * u[1])
            props.append(T.primitive([x, ground + 0.9 * e[1], z], 1.0, e, 0.0, tint, 0.0))
    ground = T.build_prop_bvh(props, leaf_size=4)
    frame.ground = ground
    frame.globals.ground_counts[:] = [len(ground), 1, 0, 0]
    land = LandscapeData(heights, terrain, cells)
    wl = Workload("terrain_1080p", frame, width, height, spp, max_bounces, {},
                  f"{cells}^2 fBm terrain, {rocks} rocks + {foliage} ellipsoids (BVH of {len(ground)} entries)", land)
    return wl, land


WORKLOADS = {
    "spheres_256": spheres_256,
    "rings_1080p": rings_1080p,
    "terrain_1080p": lambda **kw: terrain_1080p(**kw)[0],
}


def upload_workload(tracer, wl: Workload) -> None:
    """Upload a workload's extension tables (ring profiles, terrain) to a
    PathTracer or any object with the same upload methods."""
    for slot, tau in wl.ring_tables.items():
        tracer.upload_ring_profile(slot, tau)
    if wl.landscape is not None:
        if wl.landscape.detail is not None:
            tracer.upload_terrain(wl.landscape.terrain, wl.landscape.cells, wl.landscape.detail)
        else:
            tracer.upload_terrain(wl.landscape.terrain, wl.landscape.cells)
        if wl.landscape.albedo_map is not None:
            tracer.upload_albedo_map(wl.landscape.albedo_map, wl.landscape.map_extent)


def render_options(wl: Workload, spp: int = 64, noise_seed: int = 0) -> abi.Options:
    """Options for rendering a workload: `spp` samples per dispatch, the
    workload's depth, no Milky Way backdrop (no map is bound)."""
    o = abi.default_options()
    o.samples_per_frame = min(max(spp, 1), abi.MAX_BATCH_SAMPLES)
    o.max_bounces = wl.max_bounces
    o.milky_way = 0.0
    o.noise_seed = noise_seed & 0xFFFFFFFF
    return o


def earthlike_air() -> dict:
    """`Atmosphere::earthlike` (src/sim.rs:295-306): sea-level Rayleigh
    5.8, 13.5, 33.1 and Mie 21 per million metres, 8.5 km scale height,
    80 km thick, Mie asymmetry 0.76; lengths in AU."""
    return dict(scale_height=8500.0 / AU_M, thickness=80000.0 / AU_M,
                rayleigh=[5.8e-6 * AU_M, 13.5e-6 * AU_M, 33.1e-6 * AU_M], mie=21.0e-6 * AU_M, mie_g=0.76)


def with_air(frame: Frame, host_index: int, air: dict | None = None) -> Frame:
    """Give body `host_index` of a packed frame its air, as `build_frame`
    does (src/main.rs:941-962): the centre and radius of the host's packed
    sphere, the coefficients, and atmo_params.w = host index + 1."""
    a = air or earthlike_air()
    host = frame.bodies[host_index]
    g = frame.globals
    g.atmo_center[:] = [host.center[0], host.center[1], host.center[2], host.radius]
    g.atmo_rayleigh[:] = [*a["rayleigh"], a["mie"]]
    g.atmo_params[:] = [a["mie_g"], a["scale_height"], a["thickness"], float(host_index + 1)]
    return frame
