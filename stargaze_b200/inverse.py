"""The differentiable ring inverse problem and its central-difference check.

The problem: the ring-and-eclipse scene (`workloads.rings_1080p`) at
512 x 512, 64 spp per render; parameters are the ring's 512-bin optical-depth
table, its single-scattering albedo and the albedos of the bodies that do not
emit; the loss is the mean squared difference from a target image rendered
with the table perturbed by seeded Gaussian noise (sigma 0.1, clamped to
[0, 2]); Adam at lr 1e-2 runs 200 steps from the unperturbed table, each on
fresh noise. Gradients come from the path-replay adjoint through
`autograd.render`.

Only part of the table is identifiable from the image: bins the camera does
not see, or sees only through optically thick neighbours, leave the loss
unchanged. Recovery is therefore reported over the observed bins (summed
|gradient| over the first renders above a tenth of its largest value) and
over all bins.
"""
from __future__ import annotations

import time

import numpy as np

from . import workloads as W

TARGET_NOISE_SEED = 0x50000000


def perturbed_profile(base: np.ndarray, seed: int = 1, sigma: float = 0.1) -> np.ndarray:
    """The target table: `base` plus seeded N(0, sigma), clamped to [0, 2]."""
    noise = np.random.default_rng(seed).normal(0.0, sigma, base.size)
    return np.clip(base + noise, 0.0, 2.0).astype(np.float32)


def _setup(width: int, height: int, spp: int, target_spp: int, seed: int, device: int):
    import torch

    from .autograd import Renderer, render

    wl = W.rings_1080p(width, height, spp)
    base = wl.ring_tables[0]
    target_tau = perturbed_profile(base)
    ref = Renderer(wl.frame, width, height, target_spp, max_bounces=wl.max_bounces, ring_tables={0: target_tau},
                   noise_seed=TARGET_NOISE_SEED, device=device)
    with torch.no_grad():
        target = render(ref, torch.tensor(target_tau, device=f"cuda:{device}")).clone()
    ref.tracer.close()
    r = Renderer(wl.frame, width, height, spp, max_bounces=wl.max_bounces, ring_tables={0: base}, noise_seed=seed,
                 device=device)
    return wl, base, target_tau, target, r


def ring_inverse(width: int = 512, height: int = 512, spp: int = 64, steps: int = 200, lr: float = 1e-2,
                 target_spp: int = 256, seed: int = 1, device: int = 0) -> dict:
    """Runs the inverse problem; returns losses, timings and parameter errors."""
    import torch

    from .autograd import render

    wl, base, target_tau, target, r = _setup(width, height, spp, target_spp, seed, device)
    dev = torch.device("cuda", device)
    emits = torch.tensor([b.emissive >= 0.5 for b in wl.frame.bodies], device=dev)
    tau = torch.tensor(base, device=dev, requires_grad=True)
    ring_albedo0 = np.array([list(b.ring_color[:3]) for b in wl.frame.bodies], np.float32)
    body_color0 = np.array([list(b.color[:3]) for b in wl.frame.bodies], np.float32)
    ring_albedo = torch.tensor(ring_albedo0, device=dev, requires_grad=True)
    body_color = torch.tensor(body_color0, device=dev, requires_grad=True)
    opt = torch.optim.Adam([tau, ring_albedo, body_color], lr=lr)
    losses, sensitivity = [], np.zeros(base.size)
    torch.cuda.synchronize(dev)
    start = time.perf_counter()
    for step in range(steps):
        opt.zero_grad()
        loss = ((render(r, tau, ring_albedo, body_color) - target) ** 2).mean()
        loss.backward()
        with torch.no_grad():
            body_color.grad[emits] = 0.0  # emitted radiance is not a parameter here
            if step < 4:
                sensitivity += np.abs(tau.grad.cpu().numpy())
        opt.step()
        with torch.no_grad():
            tau.clamp_(0.0, 2.0)
            ring_albedo.clamp_(0.0, 1.0)
            body_color[~emits] = body_color[~emits].clamp(0.0, 1.0)
        losses.append(float(loss.detach()))
    torch.cuda.synchronize(dev)
    elapsed = time.perf_counter() - start
    r.tracer.close()
    final = tau.detach().cpu().numpy()
    observed = sensitivity > 0.1 * sensitivity.max()
    non_star = ~emits.cpu().numpy()
    return {
        "width": width, "height": height, "spp": spp, "steps": steps, "lr": lr, "bins": int(base.size),
        "parameters": int(base.size + 3 + 3 * int(non_star.sum())),
        "ms_per_step": elapsed / steps * 1e3,
        "loss_first5": float(np.mean(losses[:5])), "loss_last10": float(np.mean(losses[-10:])),
        "observed_bins": int(observed.sum()),
        "tau_error_observed": {"start": float(np.abs(base - target_tau)[observed].mean()),
                               "end": float(np.abs(final - target_tau)[observed].mean())},
        "tau_error_all": {"start": float(np.abs(base - target_tau).mean()),
                          "end": float(np.abs(final - target_tau).mean())},
        "ring_albedo_change": float(np.abs(ring_albedo.detach().cpu().numpy() - ring_albedo0).max()),
        "body_albedo_change": float(np.abs(body_color.detach().cpu().numpy() - body_color0)[non_star].max()),
    }


def directions(wl, seed: int = 7) -> dict:
    """Parameter directions of the check: three table bands and a dense
    seeded table direction (all relative to the table), the ring albedo and
    each non-emitting body's albedo."""
    tau = wl.ring_tables[0]
    n = len(wl.frame.bodies)
    out = {}
    for name, lo, hi in (("C ring", 0, 143), ("B ring", 143, 354), ("A ring", 392, 512)):
        v = np.zeros_like(tau)
        v[lo:hi] = tau[lo:hi]
        out[name] = {"tau": v}
    # Relative, so that tau - h d stays non-negative (gap bins stay at 0).
    out["dense"] = {"tau": (tau * np.random.default_rng(seed).uniform(-1.0, 1.0, tau.size)).astype(np.float32)}
    ringed = next(i for i, b in enumerate(wl.frame.bodies) if b.ring_params[0] > b.ring_plane[3])
    a = np.zeros((n, 3), np.float32)
    a[ringed] = 1.0
    out["ring albedo"] = {"ring_albedo": a}
    for i, b in enumerate(wl.frame.bodies):
        if b.emissive < 0.5:
            c = np.zeros((n, 3), np.float32)
            c[i] = b.color[:3]
            out[f"albedo {i}"] = {"body_color": c}
    return out


def central_difference_check(width: int = 512, height: int = 512, spp: int = 64, h: float = 1e-3,
                             batches: int = 6, device: int = 0) -> dict:
    """The adjoint's directional derivatives of the L2 loss against central
    differences of the same loss (step h along each direction, the same
    noise keys for both sides: common random numbers), over `batches`
    noise keys. Returns per direction the means and the standard error."""
    import torch

    from .autograd import Renderer, render

    wl, base, _target_tau, target, r = _setup(width, height, spp, 4 * spp, 11, device)
    r.tracer.close()
    dev = torch.device("cuda", device)
    ring_albedo0 = np.array([list(b.ring_color[:3]) for b in wl.frame.bodies], np.float32)
    body_color0 = np.array([list(b.color[:3]) for b in wl.frame.bodies], np.float32)

    rr = Renderer(wl.frame, width, height, spp, max_bounces=wl.max_bounces, ring_tables={0: base}, device=device)

    def loss_at(seed, tau, ra, bc, grad):
        # Noise keys from `seed` on for this render (sampling.x is the noise
        # seed plus the tracer's sequence): common random numbers.
        rr.set_noise_seed((seed - rr.tracer.sequence()) & 0xFFFFFFFF)
        t = torch.tensor(tau, device=dev, requires_grad=grad)
        a = torch.tensor(ra, device=dev, requires_grad=grad)
        c = torch.tensor(bc, device=dev, requires_grad=grad)
        loss = ((render(rr, t, a, c) - target) ** 2).mean()
        out = float(loss.detach())
        grads = None
        if grad:
            loss.backward()
            grads = (t.grad.cpu().numpy(), a.grad.cpu().numpy(), c.grad.cpu().numpy())
        return out, grads

    result = {}
    dirs = directions(wl)
    samples = {name: ([], []) for name in dirs}
    for b in range(batches):
        seed = 104729 * (b + 1)
        _, (gt, ga, gc) = loss_at(seed, base, ring_albedo0, body_color0, True)
        for name, d in dirs.items():
            dt, da, dc = d.get("tau", 0.0), d.get("ring_albedo", 0.0), d.get("body_color", 0.0)
            adj = float((gt * dt).sum() + (ga * da).sum() + (gc * dc).sum())
            lp, _ = loss_at(seed, base + h * dt, ring_albedo0 + h * da, body_color0 + h * dc, False)
            lm, _ = loss_at(seed, base - h * dt, ring_albedo0 - h * da, body_color0 - h * dc, False)
            samples[name][0].append(adj)
            samples[name][1].append((lp - lm) / (2.0 * h))
    rr.tracer.close()
    for name, (adj, fd) in samples.items():
        adj, fd = np.array(adj), np.array(fd)
        sigma = float(np.hypot(adj.std(ddof=1), fd.std(ddof=1)) / np.sqrt(len(adj)))
        result[name] = {"adjoint": float(adj.mean()), "central_difference": float(fd.mean()), "std_error": sigma,
                        "relative_difference": float(abs(adj.mean() - fd.mean()) / max(abs(fd.mean()), 1e-30))}
    return result


__all__ = ["ring_inverse", "central_difference_check", "perturbed_profile", "directions"]
