"""Batched rendering and the fused fit iteration.

* A batch of images of different sizes renders, bins and differentiates exactly as each image
  does alone (the same tile lists in the same ascending order): images and the deterministic
  gradients are bitwise equal, fast-mode gradients agree to float rounding.
* The fused fit iteration (loss + backward + moments → gradients → RS chain rule → Adam → clamp
  in our kernels) follows the eager iteration the reference runs — autograd through the
  renderer, pixel MSE, ``torch.optim.Adam`` with per-group learning rates, log-scale clamp.
* A batched fit reaches the same PSNR as fitting each image alone.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from gpu_helpers import rel_err, require_cuda
from structsplat_b200 import _native, render_gaussians
from structsplat_b200.batch import Batch, FitPlan, FitSettings, PARAM_NAMES, fit_batch
from structsplat_b200.fit import RenderPlan
from structsplat_b200.render import RECORD_FLOATS, _p, _stream
from structsplat_b200.synthetic import make_field, make_target

pytestmark = pytest.mark.gpu

SIZES = [(64, 96), (37, 50), (128, 128), (1, 1), (40, 33)]
COUNTS = [500, 120, 1500, 3, 0]


def _field(H, W, n, seed):
    f = make_field(max(H, 1), max(W, 1), n, seed=seed)
    return {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}


def _fields(sizes=SIZES, counts=COUNTS, seed=0):
    return [_field(H, W, n, seed + b) for b, ((H, W), n) in enumerate(zip(sizes, counts))]


def _batch_index(batch, params, cap=None):
    n = batch.n
    rec = torch.empty(max(n, 1) * RECORD_FLOATS, device="cuda")
    _native.call("ss_batch_project_rs", batch.ref, _p(params["means"]), _p(params["log_scales"]),
                 _p(params["rotations"]), _p(params["colors"]), _p(params["opacity_logits"]), n,
                 0.0, 3.0, _p(rec), _stream())
    wsb = _native.size_query("ss_batch_tile_index_workspace_bytes", batch.ref, n)
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    off = torch.zeros(batch.tiles + 1, dtype=torch.int32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    _native.call("ss_batch_tile_index_count", batch.ref, _p(rec), n, 0, 3.0, _p(off), _p(ws), wsb,
                 _p(status), _stream())
    total = int(off[-1])
    cap = total if cap is None else cap
    gids = torch.empty(max(cap, 1), dtype=torch.int32, device="cuda")
    _native.call("ss_batch_tile_index_fill", batch.ref, _p(rec), n, 0, 3.0, _p(off), _p(gids), cap,
                 _p(ws), wsb, _p(status), _stream())
    return rec, off, gids, cap, status


def test_batched_index_forward_backward_equal_single_images():
    require_cuda()
    fields = _fields()
    batch = Batch(SIZES, COUNTS)
    params = Batch.concat_fields(fields)
    rec, off, gids, cap, status = _batch_index(batch, params)
    P = batch.pixels
    out = torch.empty(P, 3, device="cuda")
    den = torch.empty(P, device="cuda")
    _native.call("ss_batch_render_forward", batch.ref, _p(rec), batch.n, _p(gids), cap, _p(off), 1,
                 1e-8, 0.0, _p(out), _p(den), _p(status), _stream())
    grad_out = torch.randn(P, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    grads = {}
    for det in (0, 1):
        wsb = _native.size_query("ss_render_backward_workspace_bytes", batch.n, cap, 0, 0, det)
        ws = torch.empty(max(wsb, 16), dtype=torch.uint8, device="cuda")
        g = [torch.empty(batch.n, 2, device="cuda"), torch.empty(batch.n, 3, device="cuda"),
             torch.empty(batch.n, 3, device="cuda"), torch.empty(batch.n, device="cuda")]
        _native.call("ss_batch_render_backward", batch.ref, _p(grad_out), _p(rec), batch.n,
                     _p(den), _p(out), _p(gids), cap, _p(off), 1, 1e-8, 0.0, 1, _p(g[0]),
                     _p(g[1]), _p(g[2]), _p(g[3]), det, _p(ws), wsb, _p(status), _stream())
        grads[det] = g
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    for b, (H, W) in enumerate(SIZES):
        if COUNTS[b] == 0:
            assert torch.all(out[batch.pixel_slice(b)] == 0)
            continue
        plan = RenderPlan.for_field(fields[b], H, W)
        plan_det = RenderPlan.for_field(fields[b], H, W, deterministic=True)
        go = grad_out[batch.pixel_slice(b)].view(H, W, 3).contiguous()
        plan.forward_backward(fields[b], go)
        plan_det.forward_backward(fields[b], go)
        # index: same per-tile lists, shifted by the image's first tile and first Gaussian
        t0 = int(batch.image_table[b, 3])
        T = plan.T
        lo, hi = int(off[t0]), int(off[t0 + T])
        assert torch.equal(off[t0:t0 + T + 1] - lo, plan.offsets)
        g0 = batch.gaussian_base_host[b]
        assert torch.equal(gids[lo:hi] - g0, plan.gids[: hi - lo])
        # forward: bitwise
        assert torch.equal(out[batch.pixel_slice(b)].view(H, W, 3), plan.image)
        assert torch.equal(den[batch.pixel_slice(b)].view(H, W), plan.den)
        sl = batch.gaussian_slice(b)
        ref_fast = [t.clone() for t in plan.render_input_grads(go)]
        ref_det = [t.clone() for t in plan_det.render_input_grads(go)]
        for k in range(4):
            assert torch.equal(grads[1][k][sl], ref_det[k]), k
            assert rel_err(grads[0][k][sl], ref_fast[k]) <= 1e-5, k


def test_batched_truncated_tiles_stay_exact():
    require_cuda()
    fields = _fields(seed=7)
    batch = Batch(SIZES, COUNTS)
    params = Batch.concat_fields(fields)
    rec, off, gids, cap, _ = _batch_index(batch, params)
    _, _, gids_small, small, status = _batch_index(batch, params, cap=cap // 3)
    outs = []
    for g, c in ((gids, cap), (gids_small, small)):
        out = torch.empty(batch.pixels, 3, device="cuda")
        den = torch.empty(batch.pixels, device="cuda")
        _native.call("ss_batch_render_forward", batch.ref, _p(rec), batch.n, _p(g), c, _p(off), 1,
                     1e-8, 0.0, _p(out), _p(den), None, _stream())
        outs.append(out)
    torch.cuda.synchronize()
    assert int(status.item()) & 1
    assert torch.equal(outs[0], outs[1])


def _torch_fit(field, target, iters, settings: FitSettings):
    """The reference's plain iteration in eager PyTorch around our differentiable renderer."""
    H, W, _ = target.shape
    leaves = {k: v.clone().requires_grad_(True) for k, v in field.items()}
    groups = [{"params": [leaves["means"]], "lr": settings.lr_means},
              {"params": [leaves["log_scales"]], "lr": settings.lr_scales},
              {"params": [leaves["rotations"]], "lr": settings.lr_rot},
              {"params": [leaves["colors"]], "lr": settings.lr_color},
              {"params": [leaves["opacity_logits"]], "lr": settings.lr_opacity}]
    opt = torch.optim.Adam(groups)
    lo, hi = math.log(0.35), math.log(max(H, W))
    for _ in range(iters):
        img = render_gaussians(leaves["means"], leaves["log_scales"], leaves["rotations"],
                               leaves["colors"], H, W, opacity_logits=leaves["opacity_logits"],
                               deterministic=True)
        diff = img - target
        loss = (diff * diff).mean(dim=2).mean()
        opt.zero_grad(set_to_none=False)
        loss.backward()
        opt.step()
        with torch.no_grad():
            leaves["log_scales"].clamp_(max=hi)
            leaves["log_scales"].clamp_(min=lo)
    return {k: v.detach() for k, v in leaves.items()}


@pytest.mark.parametrize("iters", [1, 8])
def test_fused_fit_step_follows_eager_torch_adam(iters):
    require_cuda()
    H, W = 72, 88
    target = torch.tensor(make_target(H, W, seed=4), device="cuda")
    field = _field(H, W, 400, seed=9)
    settings = FitSettings(deterministic=True)  # the reference's per-group learning rates
    ref = _torch_fit(field, target, iters, settings)
    mine = {k: v.clone() for k, v in field.items()}
    fit_batch([mine], [target], iters=iters, settings=settings, graph=False)
    # Adam moves each element by about lr * m / (sqrt(v) + eps) per step: where a gradient is
    # near eps (1e-8) that ratio, and so the step, swings with the last bits of the gradient.
    # The bar is therefore a fraction of the group's learning rate per element.
    lrs = dict(zip(PARAM_NAMES, settings.lrs()))
    for k in PARAM_NAMES:
        dev = float((mine[k] - ref[k]).abs().max()) / lrs[k]
        assert dev <= 2e-3, (k, dev)
        assert rel_err(mine[k], ref[k]) <= 5e-5, k


def test_batched_fit_matches_single_image_fits():
    require_cuda()
    sizes, counts = [(64, 64), (48, 80), (96, 72)], [300, 250, 500]
    targets = [torch.tensor(make_target(H, W, seed=10 + b), device="cuda")
               for b, (H, W) in enumerate(sizes)]
    settings = FitSettings(deterministic=True)
    fields = _fields(sizes, counts, seed=20)
    singles = [{k: v.clone() for k, v in f.items()} for f in fields]
    hb = fit_batch(fields, targets, iters=40, settings=settings, graph=True)
    for b in range(3):
        hs = fit_batch([singles[b]], [targets[b]], iters=40, settings=settings, graph=True)
        assert abs(hb["final_psnr"][b] - hs["final_psnr"][0]) <= 0.01
        for k in PARAM_NAMES:  # deterministic: the same arithmetic in the same order
            assert torch.equal(fields[b][k], singles[b][k]), k
    assert hb["final_psnr"][0] > 10.0


def test_graph_fit_equals_eager_fit_and_counts_steps():
    require_cuda()
    H, W = 64, 64
    target = torch.tensor(make_target(H, W, seed=2), device="cuda")
    a, b = _field(H, W, 256, seed=3), _field(H, W, 256, seed=3)
    s = FitSettings(deterministic=True)
    ha = fit_batch([a], [target], iters=25, settings=s, graph=True)
    hb = fit_batch([b], [target], iters=25, settings=s, graph=False)
    for k in PARAM_NAMES:
        assert torch.equal(a[k], b[k]), k
    assert int(ha["plan"].step_state[0]) == 25
    # the per-image loss is summed with float atomics (any order): equal to float rounding
    assert abs(ha["final_psnr"][0] - hb["final_psnr"][0]) <= 1e-4


def test_fit_replans_when_the_index_outgrows_its_capacity():
    require_cuda()
    H, W = 64, 64
    target = torch.tensor(make_target(H, W, seed=5), device="cuda")
    s = FitSettings(deterministic=True)
    a, b = _field(H, W, 300, seed=6), _field(H, W, 300, seed=6)
    batch = Batch([(H, W)], [300])
    plan = FitPlan(batch, Batch.concat_fields([a]), batch.concat_images([target]), s, capacity=64)
    plan.step()
    torch.cuda.synchronize()
    assert plan.overflowed()
    ref = fit_batch([b], [target], iters=12, settings=s, graph=False, check_every=4)
    assert ref["replans"] == 0
    import structsplat_b200.batch as B
    orig = B.FitPlan.__init__

    def tiny(self, *args, **kw):  # force a too-small first plan
        kw.setdefault("capacity", 64)
        orig(self, *args, **kw)
    B.FitPlan.__init__ = tiny
    try:
        c = _field(H, W, 300, seed=6)
        got = fit_batch([c], [target], iters=12, settings=s, graph=False, check_every=4)
    finally:
        B.FitPlan.__init__ = orig
    assert got["replans"] >= 1
    for k in PARAM_NAMES:
        assert torch.equal(c[k], b[k]), k


@pytest.mark.parametrize("loss", ["l1", "l2", "charbonnier"])
def test_fit_forward_loss_gradient_matches_autograd(loss):
    require_cuda()
    H, W = 40, 56
    target = torch.tensor(make_target(H, W, seed=8), device="cuda")
    field = _field(H, W, 200, seed=11)
    batch = Batch([(H, W)], [200])
    s = FitSettings(pixel_loss=loss)
    plan = FitPlan(batch, Batch.concat_fields([field]), batch.concat_images([target]), s)
    plan.project(); plan.count(); plan.fill()  # noqa: E702
    image = torch.empty(H * W, 3, device="cuda")
    den = torch.empty(H * W, device="cuda")
    plan.loss.zero_()
    plan.forward_loss(image=image, den=den)
    img = image.view(H, W, 3).clone().requires_grad_(True)
    diff = img - target
    if loss == "l2":
        lmap = (diff * diff).mean(dim=2)
    elif loss == "l1":
        lmap = diff.abs().mean(dim=2)
    else:
        lmap = torch.sqrt(diff * diff + 1e-3 ** 2).mean(dim=2)
    total = lmap.mean()
    (g,) = torch.autograd.grad(total, img)
    g = g.reshape(-1, 3)
    denom = den + 1e-8
    want = torch.cat([g / denom[:, None], (-(g * image).sum(1) / denom)[:, None]], 1)
    assert rel_err(plan.pixel_grad, want) <= 1e-6
    lval = float(total.detach())
    assert abs(float(plan.loss[0, 0]) - lval) <= 1e-5 * abs(lval)
    mse = float(((image.view(H, W, 3) - target) ** 2).mean())
    assert abs(float(plan.loss[0, 1]) - mse) <= 1e-5 * mse


@pytest.mark.parametrize("deterministic", [True, False])
def test_plain_fit_reaches_the_reference_psnr_trajectory(deterministic):
    """The CPU benchmark's plain fit (256², 4,096 Gaussians, 100 Adam steps at lr 1e-2, pixel
    MSE) run by the reference itself (fixture fit_plain_256_4096): every 10 steps our fused,
    graph-free iteration matches its PSNR within 0.01 dB."""
    require_cuda()
    from conftest import golden
    z = golden("fit_plain_256_4096.npz")
    H = W = 256
    target = torch.tensor(make_target(H, W, seed=int(z["seed_target"])), device="cuda")
    field = _field(H, W, 4096, seed=int(z["seed_field"]))
    batch = Batch([(H, W)], [4096])
    s = FitSettings.uniform_lr(1e-2, deterministic=deterministic)
    plan = FitPlan(batch, Batch.concat_fields([field]), batch.concat_images([target]), s)
    psnr = []
    for it in range(100):
        if it % 10 == 0:
            _, loss = plan.render()
            psnr.append(10 * math.log10(1.0 / float(loss[0, 1])))
        plan.step()
    _, loss = plan.render()
    psnr.append(10 * math.log10(1.0 / float(loss[0, 1])))
    assert not plan.overflowed()
    diff = np.abs(np.array(psnr) - z["psnr"])
    print("PSNR", np.round(psnr, 4).tolist(), "max |diff| dB", float(diff.max()))
    assert diff.max() <= 0.01
