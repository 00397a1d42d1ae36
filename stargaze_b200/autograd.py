"""torch.autograd binding of the path-replay adjoint.

`render(renderer, ring_tau, ring_albedo, body_color, albedo_map)` renders
the renderer's frame with the given material parameters and returns the
accumulated image (height, width, 3) on the renderer's CUDA device. Its
backward calls sg_backward: the forward's saved state is only the tape (the
noise keys of the accumulated samples), and the backward replays those
samples from it. Gradients are unbiased estimates of the gradient of the
expected image (see include/stargaze_b200.h, sg_backward).

Parameters (any may be None, meaning the frame's own values, no gradient):
  ring_tau     (bins,) optical-depth table of ring-table slot `tau_slot`
  ring_albedo  (bodies, 3) ring single-scattering albedo (sg_sphere.ring_color)
  body_color   (bodies, 3) albedo, or emitted radiance of an emitter
  albedo_map   (map height, map width) ground albedo texels
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import abi
from ._lib import check
from .pathtracer import PathTracer, _stream_handle
from .scene import Frame


class Renderer:
    """A PathTracer bound to a frame and a sample budget per render."""

    def __init__(self, frame: Frame, width: int, height: int, spp: int, max_bounces: int = 6,
                 ring_tables: dict | None = None, terrain=None, albedo_map=None, map_extent_m: float = 0.0,
                 tau_slot: int = 0, noise_seed: int = 0, device: int = 0):
        o = abi.default_options()
        o.samples_per_frame = min(spp, abi.MAX_BATCH_SAMPLES)
        o.sample_limit = spp
        o.max_bounces = max_bounces
        o.milky_way = 0.0
        o.noise_seed = noise_seed & 0xFFFFFFFF
        self.tracer = PathTracer((width, height), o, device=device)
        self.device = torch.device("cuda", device)
        self.frame = frame.copy()
        self.width, self.height, self.spp = width, height, spp
        self.tau_slot = tau_slot
        self.ring_tables = {k: np.asarray(v, np.float32) for k, v in (ring_tables or {}).items()}
        for slot, tau in self.ring_tables.items():
            self.tracer.upload_ring_profile(slot, tau)
        if terrain is not None:
            self.tracer.upload_terrain(terrain[0], terrain[1])
        self.map_extent = map_extent_m
        self.albedo_map = None if albedo_map is None else np.asarray(albedo_map, np.float32)
        if self.albedo_map is not None:
            self.tracer.upload_albedo_map(self.albedo_map, map_extent_m)

    def set_noise_seed(self, seed: int) -> None:
        self.tracer.update_options(noise_seed=seed & 0xFFFFFFFF)

    def _apply(self, ring_tau, ring_albedo, body_color, albedo_map) -> Frame:
        frame = self.frame.copy()
        if ring_tau is not None:
            tau = ring_tau.detach().float().cpu().numpy()
            self.tracer.upload_ring_profile(self.tau_slot, tau)
        if ring_albedo is not None:
            ra = ring_albedo.detach().float().cpu().numpy()
            for i, b in enumerate(frame.bodies):
                b.ring_color[0], b.ring_color[1], b.ring_color[2] = (float(v) for v in ra[i])
        if body_color is not None:
            bc = body_color.detach().float().cpu().numpy()
            for i, b in enumerate(frame.bodies):
                b.color[0], b.color[1], b.color[2] = (float(v) for v in bc[i])
        if albedo_map is not None:
            self.tracer.upload_albedo_map(albedo_map.detach().float().cpu().numpy(), self.map_extent)
        return frame

    def forward(self, ring_tau, ring_albedo, body_color, albedo_map):
        """Render spp fresh samples; returns (image (h, w, 4), frame, tape)."""
        frame = self._apply(ring_tau, ring_albedo, body_color, albedo_map)
        stream = torch.cuda.current_stream(self.device)
        # A fresh accumulation: the history key changes with the frame; a
        # re-render of identical parameters continues the noise sequence,
        # so force a restart through the scene time.
        frame.scene_time = float(self.tracer.sequence())
        while True:
            self.tracer.encode(frame, stream)
            if self.tracer.samples() >= self.spp:
                break
        image = torch.empty((self.height, self.width, 4), dtype=torch.float32, device=self.device)
        lib = self.tracer._lib
        check(lib.sg_read_accumulation(self.tracer.handle, C.c_void_p(image.data_ptr()), 1, _stream_handle(stream)),
              self.tracer.handle)
        return image, frame, self.tracer.tape()

    def backward(self, frame: Frame, tape: abi.Tape, grad_image: torch.Tensor):
        """d loss / d parameters for d loss / d image = grad_image (h, w, 3)."""
        n = len(frame.bodies)
        dl = torch.zeros((self.height, self.width, 4), dtype=torch.float32, device=self.device)
        dl[..., :3] = grad_image.to(self.device, torch.float32)
        out = {
            "ring_tau": torch.zeros((abi.RING_TABLE_SLOTS, abi.RING_TABLE_MAX_BINS), dtype=torch.float32,
                                    device=self.device),
            "ring_albedo": torch.zeros((max(n, 1), 3), dtype=torch.float32, device=self.device),
            "body_color": torch.zeros((max(n, 1), 3), dtype=torch.float32, device=self.device),
            "albedo_map": None,
        }
        if self.albedo_map is not None:
            out["albedo_map"] = torch.zeros(self.albedo_map.shape, dtype=torch.float32, device=self.device)
        g = abi.Gradients(out["ring_tau"].data_ptr(), out["ring_albedo"].data_ptr(), out["body_color"].data_ptr(),
                          out["albedo_map"].data_ptr() if out["albedo_map"] is not None else None, 0)
        view = frame.view()
        stream = torch.cuda.current_stream(self.device)
        lib = self.tracer._lib
        check(lib.sg_backward(self.tracer.handle, C.byref(view), C.byref(tape), C.c_void_p(dl.data_ptr()), 1,
                              C.byref(g), _stream_handle(stream)), self.tracer.handle)
        out["dropped"] = int(g.dropped)
        out["ring_albedo"] = out["ring_albedo"][:n]
        out["body_color"] = out["body_color"][:n]
        return out


class _Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, renderer: Renderer, ring_tau, ring_albedo, body_color, albedo_map):
        image, frame, tape = renderer.forward(ring_tau, ring_albedo, body_color, albedo_map)
        ctx.renderer, ctx.frame, ctx.tape = renderer, frame, tape
        ctx.bins = None if ring_tau is None else ring_tau.numel()
        return image[..., :3]

    @staticmethod
    def backward(ctx, grad_image):
        r = ctx.renderer
        g = r.backward(ctx.frame, ctx.tape, grad_image.contiguous())
        tau = None if ctx.bins is None else g["ring_tau"][r.tau_slot, : ctx.bins]
        needs = ctx.needs_input_grad
        return (None,
                tau if needs[1] else None,
                g["ring_albedo"] if needs[2] else None,
                g["body_color"] if needs[3] else None,
                g["albedo_map"] if needs[4] else None)


def render(renderer: Renderer, ring_tau=None, ring_albedo=None, body_color=None, albedo_map=None) -> torch.Tensor:
    """Differentiable render: (height, width, 3) image on the CUDA device."""
    return _Render.apply(renderer, ring_tau, ring_albedo, body_color, albedo_map)


__all__ = ["Renderer", "render"]
