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


def spheres_256(width: int = 256, height: int = 256, spp: int = 64) -> Workload:
    star = Body(np.array([1.5e11, 0.0, 0.0]), 7.0e8, luminosity_w=3.8e26)
    host = Body(np.zeros(3), 6.4e6, albedo=(0.3, 0.3, 0.3))
    moon_dir = np.array([math.cos(math.radians(100.0)), math.sin(math.radians(100.0)), 0.0])
    moon = Body(3.84e8 * moon_dir, 1.74e6, albedo=(0.12, 0.12, 0.12))
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
    moon = Body(planet_pos + 2.0e8 * moon_dir, 1.5e6, albedo=(0.12, 0.12, 0.12))
    pole = np.array([0.3, 0.2, 0.93])
    ring = Ring(7.4e7, 1.37e8, (0.5, 0.5, 0.5), optical_depth=1.0, table_slot=0, pole=pole / np.linalg.norm(pole))
    planet = Body(planet_pos, 5.8e7, albedo=(0.5, 0.5, 0.5), ring=ring)
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


WORKLOADS = {"spheres_256": spheres_256, "rings_1080p": rings_1080p}


def render_options(wl: Workload, spp: int = 64, noise_seed: int = 0) -> abi.Options:
    """Options for rendering a workload: `spp` samples per dispatch, the
    workload's depth, no Milky Way backdrop (no map is bound)."""
    o = abi.default_options()
    o.samples_per_frame = min(max(spp, 1), abi.MAX_BATCH_SAMPLES)
    o.max_bounces = wl.max_bounces
    o.milky_way = 0.0
    o.noise_seed = noise_seed & 0xFFFFFFFF
    return o
