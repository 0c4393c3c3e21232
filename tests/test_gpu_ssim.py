"""The SSIM term of the fit loss on the GPU (ss_ssim_target_stats, ss_fit_ssim).

* Value and gradient w.r.t. the rendered image against the reference's metrics.ssim
  (tests/golden/ssim_*.npz), all fixture images in one batch (per-image windows and means).
* The mixed loss (1 - w) pixel_loss + w (1 - SSIM) of the fit loop (fit.py:3244) through the
  normalisation, against torch autograd of the oracle on the rendered image.
* A fit with the SSIM term follows the eager iteration: render, autograd through the oracle's
  mixed loss, torch.optim.Adam, log-scale clamp.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest
import torch

from gpu_helpers import rel_err, require_cuda
from oracle import ssim_ref
from structsplat_b200 import _native
from structsplat_b200.batch import Batch, FitPlan, FitSettings, PARAM_NAMES
from structsplat_b200.render import _p, _stream
from structsplat_b200.synthetic import make_field, make_target

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("ssim_*.npz"))


def _ssim_grad(batch, image, target, weight=1.0, normalize=0, den=None, eps=1e-8,
               pixel_grad=None):
    P = batch.pixels
    wsb = _native.size_query("ss_ssim_workspace_bytes", P)
    ws = torch.empty(max(wsb // 4, 1), device="cuda")
    stats = torch.empty(6 * P, device="cuda")
    _native.call("ss_ssim_target_stats", batch.ref, _p(target), _p(stats), _p(ws), wsb,
                 _stream())
    pg = torch.zeros(P, 4, device="cuda") if pixel_grad is None else pixel_grad
    ssim = torch.zeros(batch.images, device="cuda")
    _native.call("ss_fit_ssim", batch.ref, _p(image), _p(den), _p(target), _p(stats),
                 int(normalize), float(eps), float(weight), _p(pg), _p(ssim), _p(ws), wsb,
                 _stream())
    torch.cuda.synchronize()
    return pg, ssim


def test_ssim_value_and_gradient_match_the_reference():
    require_cuda()
    zs = [np.load(GOLDEN / f"{n}.npz") for n in CASES]
    sizes = [z["pred"].shape[:2] for z in zs]
    batch = Batch(sizes, [0] * len(zs))
    image = torch.tensor(np.concatenate([z["pred"].reshape(-1, 3) for z in zs]), device="cuda")
    target = torch.tensor(np.concatenate([z["target"].reshape(-1, 3) for z in zs]),
                          device="cuda")
    for _ in range(2):  # the second call reuses the workspace
        pg, ssim = _ssim_grad(batch, image, target)
        base = 0
        for b, z in enumerate(zs):
            H, W = z["pred"].shape[:2]
            assert abs(float(ssim[b]) - float(z["ssim"])) <= 2e-6
            got = -pg[base:base + H * W, :3].cpu().numpy().reshape(H, W, 3)
            assert np.abs(got - z["grad_ssim"]).max() <= 1e-4 * np.abs(z["grad_ssim"]).max()
            assert float(pg[base:base + H * W, 3].abs().max()) == 0.0
            base += H * W


@pytest.mark.parametrize("normalize", [True, False])
def test_mixed_loss_pixel_grad_matches_autograd(normalize):
    require_cuda()
    H, W = 40, 56
    target = torch.tensor(make_target(H, W, seed=8), device="cuda")
    f = make_field(H, W, 300, seed=11)
    field = {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}
    batch = Batch([(H, W)], [300])
    w = 0.3
    s = FitSettings(pixel_loss="l1", ssim_weight=w, normalize=normalize)
    plan = FitPlan(batch, Batch.concat_fields([field]), batch.concat_images([target]), s)
    plan.project(); plan.count(); plan.fill()  # noqa: E702
    plan.loss.zero_()
    plan.ssim.zero_()
    plan.forward_loss(image=plan.image, den=plan.den)
    plan.ssim_term()
    torch.cuda.synchronize()
    img = plan.image.view(H, W, 3).clone().requires_grad_(True)
    loss = ssim_ref.mixed_loss(img, target, w, "l1")
    (g,) = torch.autograd.grad(loss, img)
    g = g.reshape(-1, 3)
    if normalize:
        d = plan.den + s.eps
        want = torch.cat([g / d[:, None], (-(g * plan.image).sum(1) / d)[:, None]], 1)
    else:
        want = torch.cat([g, torch.zeros_like(g[:, :1])], 1)
    assert rel_err(plan.pixel_grad, want) <= 1e-4
    # the value only feeds reporting: float32 cancellation in E[p^2] - mu_p^2, evaluated in
    # another order than torch's convolutions, moves it by ~1e-5
    s_val = float(ssim_ref.ssim(plan.image.view(H, W, 3), target))
    assert abs(float(plan.ssim[0]) - s_val) <= 2e-5


@pytest.mark.parametrize("deterministic", [False, True])
def test_ssim_fit_follows_the_eager_iteration(deterministic):
    """Three steps of the plan against render -> oracle mixed loss -> autograd -> Adam -> clamp
    in torch, from the same field."""
    require_cuda()
    from structsplat_b200 import render_gaussians
    H, W = 48, 40
    target = torch.tensor(make_target(H, W, seed=21), device="cuda")
    f = make_field(H, W, 250, seed=22)
    w, lr = 0.3, 1e-2
    s = FitSettings.uniform_lr(lr, pixel_loss="l1", ssim_weight=w, deterministic=deterministic)
    field = {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}
    batch = Batch([(H, W)], [250])
    plan = FitPlan(batch, Batch.concat_fields([field]), batch.concat_images([target]), s)
    leaves = [torch.tensor(getattr(f, k), device="cuda").requires_grad_(True) for k in PARAM_NAMES]
    opt = torch.optim.Adam(leaves, lr=lr, betas=s.betas, eps=s.adam_eps)
    lo, hi = math.log(s.scale_min), math.log(max(H, W))
    for _ in range(3):
        plan.step()
        img = render_gaussians(*leaves[:4], H, W, opacity_logits=leaves[4],
                               normalize=s.normalize, eps=s.eps)
        loss = ssim_ref.mixed_loss(img, target, w, "l1")
        opt.zero_grad()
        loss.backward()
        opt.step()
        with torch.no_grad():
            leaves[1].clamp_(max=hi).clamp_(min=lo)
    torch.cuda.synchronize()
    for k, leaf in zip(PARAM_NAMES, leaves):
        diff = float((plan.params[k] - leaf.detach()).abs().max())
        assert diff <= 2e-3 * lr, (k, diff)


def test_tile_passes_equal_the_per_pixel_passes():
    """Tile sizes 16 and 32 stage each tile with its halo in shared memory; other tile sizes
    run the per-pixel passes.  Same taps in the same order: the same gradient to float rounding
    (the compiler may fuse a product into an FMA in one form and not the other)."""
    require_cuda()
    sizes = [(70, 45), (33, 64), (5, 7)]
    rng = np.random.default_rng(3)
    target = torch.tensor(np.concatenate([make_target(H, W, seed=b).reshape(-1, 3)
                                          for b, (H, W) in enumerate(sizes)]), device="cuda")
    image = (target + torch.tensor(rng.normal(0, 0.1, target.shape), dtype=torch.float32,
                                   device="cuda")).clamp(0, 1).contiguous()
    den = torch.tensor(rng.uniform(0.5, 2.0, target.shape[0]), dtype=torch.float32, device="cuda")
    out = {}
    for ts in (8, 16, 32):
        batch = Batch(sizes, [0] * len(sizes), tile_size=ts)
        pg0 = torch.tensor(rng.normal(0, 1e-3, (target.shape[0], 4)), dtype=torch.float32,
                           device="cuda") if ts == 8 else out[8][2].clone()
        pg, ssim = _ssim_grad(batch, image, target, weight=0.3, normalize=1, den=den,
                              pixel_grad=pg0.clone())
        out[ts] = (pg, ssim, pg0)
    for ts in (16, 32):
        assert rel_err(out[ts][0], out[8][0]) <= 1e-6, ts
        assert float((out[ts][1] - out[8][1]).abs().max()) <= 1e-6
