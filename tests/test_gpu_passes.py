"""Activity, coverage and raw weight map on the GPU against the reference (fixtures pass_*).

Bars: activity and the raw weight map within 1e-5 relative (float32 SFU exponent), their
RS-parameter gradients within 1e-4 relative; coverage from one forward equals the render's
own denominator bitwise.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import rel_err, require_cuda
from oracle import field_ref
from structsplat_b200 import render as R
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu
CASES = golden_names("pass_")


@pytest.mark.parametrize("name", CASES)
def test_activity_matches_reference(name):
    require_cuda()
    z = golden(name)
    a = float(z["fade_alpha"])
    act = R.gaussian_activity(torch.tensor(z["means"], device="cuda"),
                              torch.tensor(z["conics"], device="cuda"),
                              torch.tensor(z["radii"], device="cuda"), int(z["H"]), int(z["W"]),
                              support_fade=a > 0, support_fade_alpha=a)
    want = z["activity"]
    err = np.abs(act.cpu().numpy() - want) / np.maximum(np.abs(want), 1e-3 * np.abs(want).max())
    assert err.max() <= 1e-5


def test_activity_is_deterministic_and_lane_split_independent():
    require_cuda()
    f = make_field(256, 256, 5000, seed=4)
    m = torch.tensor(f.means, device="cuda")
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    c = field_ref.conics(ls, rot).cuda().contiguous()
    r = field_ref.radii(ls, rot, 3.0).cuda().contiguous()
    a1 = R.gaussian_activity(m, c, r, 256, 256)
    a2 = R.gaussian_activity(m, c, r, 256, 256)
    assert torch.equal(a1, a2)
    from oracle import render_ref
    ref = render_ref.activity(m.cpu().double(), c.cpu().double(), r.cpu(), 256, 256)
    assert rel_err(a1, ref) <= 1e-5


@pytest.mark.parametrize("name", CASES)
def test_raw_weight_map_and_gradients_match_reference(name):
    require_cuda()
    z = golden(name)
    H, W, a = int(z["H"]), int(z["W"]), float(z["fade_alpha"])
    p = {k: torch.tensor(z[k], device="cuda").requires_grad_(True)
         for k in ("means", "log_scales", "rotations", "opacity_logits")}
    conics = field_ref.conics(p["log_scales"], p["rotations"])
    radii = field_ref.radii(p["log_scales"].detach(), p["rotations"].detach(), 3.0)
    den = R.raw_weight_map(p["means"], conics, radii, H, W,
                           opacities=torch.sigmoid(p["opacity_logits"]), support_fade=a > 0,
                           support_fade_alpha=a)
    assert rel_err(den, z["den"]) <= 1e-5
    grads = torch.autograd.grad((den * torch.tensor(z["G"], device="cuda")).sum(), list(p.values()))
    for k, g in zip(p, grads):
        assert rel_err(g, z[f"g_{k}"]) <= 1e-4, k


def test_coverage_equals_render_denominator():
    require_cuda()
    f = make_field(96, 80, 700, seed=6)
    m = torch.tensor(f.means, device="cuda")
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    c = field_ref.conics(ls, rot).cuda().contiguous()
    r = field_ref.radii(ls, rot, 3.0).cuda().contiguous()
    col = torch.tensor(f.colors, device="cuda")
    op = torch.sigmoid(torch.tensor(f.opacity_logits, device="cuda"))
    out, den = R.render_cuda_exact_with_coverage(m, c, col, r, 96, 80, opacities=op)
    img = R.render_b200(m, c, col, r, 96, 80, opacities=op)
    assert torch.equal(out, img)
    rw = R.raw_weight_map(m, c, r, 96, 80, opacities=op)
    assert torch.equal(rw.view(96, 80), den)
