"""The fused fit tile pass (``ss_fit_forward_backward``: forward, pixel loss and backward of a
tile in one CTA) against the two-kernel step it replaces (``ss_fit_forward_loss`` then
``ss_fit_backward``).

* The image and den are bitwise those of the forward kernel (the same per-pixel order over the
  same staged records), the per-image loss agrees to float-atomic rounding.
* Deterministic mode: the per-entry moment partials and their by-Gaussian order are bitwise
  equal, so a fused fit follows the two-kernel fit bitwise.  Fast mode: the moments agree to
  the rounding of their float atomics.
* Tile lists longer than the shared-memory stage (streamed twice: once for the forward, once
  for the backward) and both tile sizes are covered.
"""
from __future__ import annotations

import pytest
import torch

from gpu_helpers import rel_err, require_cuda
from structsplat_b200 import _native
from structsplat_b200.batch import LOSS_KINDS, Batch, FitPlan, FitSettings, PARAM_NAMES, fit_batch
from structsplat_b200.render import _p, _stream
from structsplat_b200.synthetic import make_field, make_target

pytestmark = pytest.mark.gpu

SIZES = [(64, 96), (37, 50), (1, 1), (128, 128), (40, 33), (20, 17)]
COUNTS = [500, 120, 3, 1500, 60, 0]  # a one-pixel image and an image without Gaussians


def _fields(sizes, counts, seed, log_sigma_std=0.5):
    out = []
    for b, ((H, W), n) in enumerate(zip(sizes, counts)):
        f = make_field(H, W, n, seed=seed + b, log_sigma_std=log_sigma_std)
        out.append({k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES})
    return out


def _plans(sizes, counts, settings, ts, seed=0, log_sigma_std=0.5):
    """Two plans over identical fields, one per path, with their tile indices built."""
    targets = [torch.tensor(make_target(H, W, seed=40 + b), device="cuda")
               for b, (H, W) in enumerate(sizes)]
    plans = []
    for fused in (True, False):
        s = FitSettings(**{**settings.__dict__, "fused": fused})
        fields = _fields(sizes, counts, seed, log_sigma_std)
        batch = Batch(sizes, counts, tile_size=ts)
        plan = FitPlan(batch, Batch.concat_fields(fields), batch.concat_images(targets), s)
        plan.project()
        plan.count()
        plan.fill()
        plans.append(plan)
    return plans


def _fused_call(plan, image, den):
    s = plan.s
    _native.call("ss_fit_forward_backward", plan.batch.ref, _p(plan.records), plan.n,
                 _p(plan.gids), plan.capacity, _p(plan.offsets), int(s.normalize), float(s.eps),
                 float(plan.tail), _p(plan.target), LOSS_KINDS[s.pixel_loss],
                 float(s.charbonnier_eps), _p(image), _p(den), _p(plan.loss),
                 int(s.deterministic), _p(plan.bwd_ws), plan.bwd_ws_bytes, _p(plan.status),
                 _stream())


def _compare(plans, deterministic):
    fused, plain = plans
    P = fused.batch.pixels
    img = [torch.full((P, 3), -1.0, device="cuda") for _ in range(2)]
    den = [torch.full((P,), -1.0, device="cuda") for _ in range(2)]
    for p in plans:
        p.loss.zero_()
        p.bwd_ws.zero_()
    _fused_call(fused, img[0], den[0])
    plain.forward_loss(image=img[1], den=den[1])
    plain.backward()
    torch.cuda.synchronize()
    assert not fused.overflowed() and not plain.overflowed()
    assert torch.equal(img[0], img[1])
    assert torch.equal(den[0], den[1])
    assert rel_err(fused.loss, plain.loss) <= 1e-5
    n, cap = fused.n, fused.capacity
    if deterministic:
        # partials (cap x 12 floats), sort keys and entry order (4 x cap ints), run bounds (2n)
        a256 = lambda b: (b + 255) // 256 * 256
        fixed = (a256(48 * cap) + 4 * a256(4 * cap) + a256(8 * n)) // 4
        assert torch.equal(fused.bwd_ws[:fixed], plain.bwd_ws[:fixed])
    else:
        assert rel_err(fused.bwd_ws[: 9 * n], plain.bwd_ws[: 9 * n]) <= 1e-5


@pytest.mark.parametrize("deterministic", [True, False])
@pytest.mark.parametrize("loss", ["l2", "l1", "charbonnier"])
def test_fused_pass_equals_two_kernels(loss, deterministic):
    require_cuda()
    s = FitSettings(pixel_loss=loss, deterministic=deterministic)
    _compare(_plans(SIZES, COUNTS, s, ts=32), deterministic)


@pytest.mark.parametrize("ts", [16, 32])
@pytest.mark.parametrize("normalize,fade", [(True, 0.0), (False, 0.0), (True, 0.5)])
def test_fused_pass_modes_and_tile_sizes(ts, normalize, fade):
    require_cuda()
    s = FitSettings(normalize=normalize, fade_alpha=fade, deterministic=True)
    _compare(_plans(SIZES, COUNTS, s, ts=ts, seed=7), True)


@pytest.mark.parametrize("ts", [16, 32])
def test_fused_pass_streams_long_tile_lists(ts):
    """Lists longer than the stage (448 / 512 records) are streamed once per phase."""
    require_cuda()
    s = FitSettings(deterministic=True)
    plans = _plans([(64, 64)], [6000], s, ts=ts, seed=11, log_sigma_std=0.9)
    counts = plans[0].offsets[1:] - plans[0].offsets[:-1]
    assert int(counts.max()) > 512  # the streamed path runs
    _compare(plans, True)


def test_fused_fit_follows_the_two_kernel_fit():
    require_cuda()
    sizes, counts = [(64, 64), (48, 80)], [300, 250]
    targets = [torch.tensor(make_target(H, W, seed=60 + b), device="cuda")
               for b, (H, W) in enumerate(sizes)]
    runs = []
    for fused in (True, False):
        fields = _fields(sizes, counts, seed=70)
        s = FitSettings(deterministic=True, fused=fused)
        h = fit_batch(fields, targets, iters=20, settings=s, graph=True)
        runs.append((fields, h))
    (fa, ha), (fb, hb) = runs
    for b in range(len(sizes)):
        for k in PARAM_NAMES:
            assert torch.equal(fa[b][k], fb[b][k]), k
        assert abs(ha["final_psnr"][b] - hb["final_psnr"][b]) <= 1e-4
