"""The fused render forward + backward (``ss_render_forward_backward``, used by
``RenderPlan.forward_backward`` in a plan built with ``fused=True``) against the forward and
backward tile kernels one after the other, on identical plans.

* The image and den are bitwise the forward kernel's (the same per-pixel order over the same
  staged records), and the backward's pixel inputs repeat the backward kernel's arithmetic.
* Deterministic mode: the gradients are bitwise equal.  Fast mode: they agree to the rounding
  of the moments' float atomics.
* Normalised and additive modes, both tile sizes, tile lists longer than the shared-memory
  stage, tiles truncated by the capacity (they scan every Gaussian in both paths), a one-pixel
  image and a field without Gaussians.
"""
from __future__ import annotations

import pytest
import torch

from gpu_helpers import rel_err, require_cuda
from structsplat_b200.fit import PARAM_NAMES, RenderPlan
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu

CASES = [  # H, W, Gaussians, log-sigma spread
    (64, 96, 500, 0.5),
    (37, 50, 120, 0.5),
    (1, 1, 3, 0.5),
    (80, 72, 3000, 1.0),  # tile lists longer than the stage
    (40, 33, 0, 0.5),
]


def _field(H, W, n, std, seed):
    f = make_field(H, W, n, seed=seed, log_sigma_std=std)
    return {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}


def _run(params, grad_out, H, W, fused, capacity=None, **kw):
    if capacity is None:
        plan = RenderPlan.for_field(params, H, W, fused=fused, **kw)
    else:
        plan = RenderPlan(n=params["means"].shape[0], H=H, W=W, capacity=capacity, fused=fused,
                          device=params["means"].device, **kw)
    grads = plan.forward_backward(params, grad_out)
    torch.cuda.synchronize()
    return plan, {k: v.clone() for k, v in grads.items()}


@pytest.mark.parametrize("tile_size", [16, 32])
@pytest.mark.parametrize("normalize", [True, False])
@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("case", CASES)
def test_fused_render_matches_the_two_kernel_step(case, deterministic, normalize, tile_size):
    require_cuda()
    H, W, n, std = case
    params = _field(H, W, n, std, seed=H * 7 + n)
    grad_out = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    kw = dict(normalize=normalize, deterministic=deterministic, tile_size=tile_size)
    a, ga = _run(params, grad_out, H, W, True, **kw)
    b, gb = _run(params, grad_out, H, W, False, **kw)
    assert a.use_fused() and not b.use_fused()
    assert torch.equal(a.image, b.image)
    assert torch.equal(a.den, b.den)
    assert int(a.status.item()) == int(b.status.item()) == 0
    for k in ga:
        if deterministic:
            assert torch.equal(ga[k], gb[k]), k
        else:
            assert rel_err(ga[k], gb[k]) <= 1e-5, k


def test_fused_pass_is_opt_in():
    require_cuda()
    params = _field(32, 32, 10, 0.5, seed=1)
    assert not RenderPlan.for_field(params, 32, 32).use_fused()
    assert RenderPlan.for_field(params, 32, 32, fused=True).use_fused()


def test_truncated_tiles_render_exactly_in_the_fused_pass():
    """A capacity below the tile-list total: truncated tiles scan every Gaussian in ascending
    id, in the fused pass as in the forward kernel, and the overflow is raised in both."""
    require_cuda()
    H, W, n = 96, 80, 800
    params = _field(H, W, n, 0.7, seed=3)
    grad_out = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(9))
    a, ga = _run(params, grad_out, H, W, True, capacity=500)
    b, gb = _run(params, grad_out, H, W, False, capacity=500)
    full, gf = _run(params, grad_out, H, W, False)
    assert a.overflowed() and b.overflowed() and not full.overflowed()
    assert torch.equal(a.image, b.image)
    assert torch.equal(a.image, full.image)
    # fast mode: the moments are float atomics, so the three runs agree to their rounding
    # (about 1e-5 of the gradient's scale on this 800-Gaussian field)
    for k in ga:
        assert rel_err(ga[k], gb[k]) <= 5e-5, k
        assert rel_err(ga[k], gf[k]) <= 5e-5, k


def test_fused_render_gradients_match_autograd():
    """The fused step against torch autograd of the eager renderer (render_gaussians)."""
    require_cuda()
    from structsplat_b200 import render_gaussians
    H, W, n = 48, 64, 400
    params = _field(H, W, n, 0.5, seed=17)
    grad_out = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    plan, g = _run(params, grad_out, H, W, True)
    leaves = [params[k].clone().requires_grad_(True) for k in PARAM_NAMES]
    img = render_gaussians(*leaves[:4], H, W, opacity_logits=leaves[4])
    want = torch.autograd.grad(img, leaves, grad_out)
    assert torch.equal(plan.image, img.detach())
    for k, w in zip(PARAM_NAMES, want):
        assert rel_err(g[k], w) <= 1e-5, k
