"""The torch.autograd binding of the adjoint (stargaze_b200.autograd) and the
ring inverse problem it serves (a reduced form of the differentiable ring
workload: recover a perturbed optical-depth profile with Adam)."""
import numpy as np
import pytest

from stargaze_b200 import workloads as W
from stargaze_b200.pathtracer import PathTracer

pytestmark = pytest.mark.gpu

WIDTH = HEIGHT = 128
BINS = 32


def coarse_profile() -> np.ndarray:
    """The ring workload's 512-bin profile averaged down to BINS bins."""
    return W.ring_tau_profile(512, seed=0).reshape(BINS, -1).mean(axis=1).astype(np.float32)


def renderer(spp: int, seed: int = 0):
    from stargaze_b200.autograd import Renderer

    wl = W.rings_1080p(WIDTH, HEIGHT, spp)
    return wl, Renderer(wl.frame, WIDTH, HEIGHT, spp, max_bounces=wl.max_bounces,
                        ring_tables={0: coarse_profile()}, noise_seed=seed)


def test_autograd_gradients_equal_sg_backward():
    import torch

    from stargaze_b200.autograd import render

    wl, r = renderer(16, seed=7)
    tau = torch.tensor(coarse_profile(), device="cuda", requires_grad=True)
    ring_albedo = torch.tensor([list(b.ring_color[:3]) for b in wl.frame.bodies], device="cuda",
                               requires_grad=True)
    body_color = torch.tensor([list(b.color[:3]) for b in wl.frame.bodies], device="cuda", requires_grad=True)
    image = render(r, tau, ring_albedo, body_color)
    assert image.shape == (HEIGHT, WIDTH, 3)
    weights = torch.rand((HEIGHT, WIDTH, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    (image * weights).sum().backward()
    # The same samples through the plain C ABI: the renderer's first frame
    # starts the noise sequence at 0 with scene time 0.
    t = PathTracer((WIDTH, HEIGHT), W.render_options(wl, 16, noise_seed=7))
    t.upload_ring_profile(0, coarse_profile())
    frame = wl.frame.copy()
    frame.scene_time = 0.0
    t.encode(frame)
    np.testing.assert_allclose(t.read_pixels()[:, :3].reshape(HEIGHT, WIDTH, 3), image.detach().cpu().numpy(),
                               rtol=0, atol=0)
    dl = np.zeros((HEIGHT * WIDTH, 4), np.float32)
    dl[:, :3] = weights.cpu().numpy().reshape(-1, 3)
    g = t.backward(frame, t.tape(), dl)
    np.testing.assert_allclose(tau.grad.cpu().numpy(), g.ring_tau[0, :BINS], rtol=1e-4,
                               atol=1e-6 * float(np.abs(g.ring_tau).max()))
    np.testing.assert_allclose(ring_albedo.grad.cpu().numpy(), g.ring_albedo, rtol=1e-4, atol=1e-9)
    np.testing.assert_allclose(body_color.grad.cpu().numpy(), g.body_color, rtol=1e-4, atol=1e-9)
    assert g.dropped == 0


def test_adam_recovers_a_perturbed_ring_profile():
    """Target: the profile plus seeded Gaussian noise (sigma 0.1, clamped to
    [0, 2]); start: the unperturbed profile; L2 image loss against a 256-spp
    target; Adam, lr 1e-2, 60 steps of 32 spp. The bins the image depends on
    (start gradient above 10 % of the largest, averaged over four renders)
    must be recovered; optically thick or unseen bins are not identifiable
    from the image and are left out."""
    import torch

    from stargaze_b200.autograd import render

    base = coarse_profile()
    target_tau = np.clip(base + np.random.default_rng(3).normal(0.0, 0.1, BINS), 0.0, 2.0).astype(np.float32)
    _, ref = renderer(256, seed=99)
    with torch.no_grad():
        target = render(ref, torch.tensor(target_tau, device="cuda")).clone()
    _, r = renderer(32, seed=1)
    tau = torch.tensor(base, device="cuda", requires_grad=True)
    sensitivity = np.zeros(BINS)
    for _ in range(4):
        tau.grad = None
        ((render(r, tau) - target) ** 2).sum().backward()
        sensitivity += np.abs(tau.grad.cpu().numpy())
    observed = sensitivity > 0.1 * sensitivity.max()
    assert observed.sum() >= 6
    error0 = float(np.abs(base - target_tau)[observed].mean())
    opt = torch.optim.Adam([tau], lr=1e-2)
    losses = []
    for _ in range(60):
        opt.zero_grad()
        loss = ((render(r, tau) - target) ** 2).sum()
        loss.backward()
        opt.step()
        with torch.no_grad():
            tau.clamp_(0.0, 2.0)
        losses.append(float(loss.detach()))
    error = float(np.abs(tau.detach().cpu().numpy() - target_tau)[observed].mean())
    assert np.mean(losses[-10:]) < 0.8 * np.mean(losses[:5]), losses
    assert error < 0.4 * error0, (error0, error)
