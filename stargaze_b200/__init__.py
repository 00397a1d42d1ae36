"""stargaze_b200 — B200 (sm_100a) progressive path-tracing integrator.

A drop-in for the wgpu compute pass of stargaze's `PathTracer`
(src/pathtracer.rs): the same packed scene buffers (`Settings`, `Globals`,
`Sphere`, `Primitive`) and the same progressive accumulation contract, with
the integrator running as hand-written CUDA kernels behind a C ABI
(include/stargaze_b200.h).
"""
from . import abi
from ._lib import StargazeError, load
from .pathtracer import HIT_DTYPE, RAY_DTYPE, PathTracer, rays_array
from .scene import Frame, body, frame, ringed

__all__ = [
    "abi",
    "load",
    "StargazeError",
    "PathTracer",
    "Frame",
    "frame",
    "body",
    "ringed",
    "rays_array",
    "RAY_DTYPE",
    "HIT_DTYPE",
]
