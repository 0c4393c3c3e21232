"""FP64 central finite differences pin the analytic gradient the GPU path is measured against.

Sub-case of the fwd+bwd benchmark: 64x64 image, 256 Gaussians from the benchmark field
distribution, normalized and additive modes.  L = sum(image * G) for a fixed random G; the
float64 oracle's autograd gradient w.r.t. the RS field parameters (means, log-scales,
rotations, colours, opacity logits) is compared with central differences of L at step 1e-4 on
a seeded sample of parameters.  A mean perturbation that moves the rounded centre (and so the
clipped support rectangle) makes L discontinuous; such coordinates are skipped.  The GPU
gradients are then compared with this same float64 gradient (tests/test_gpu_render.py and the
golden cases), which closes the chain GPU -> float64 analytic -> finite differences.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import field_ref, render_ref
from structsplat_b200.synthetic import make_field

H = W = 64
N = 256
STEP = 1e-4
NAMES = ("means", "log_scales", "rotations", "colors", "opacity_logits")


def _loss(p, G, normalize):
    conics = field_ref.conics(p["log_scales"], p["rotations"])
    radii = field_ref.radii(p["log_scales"], p["rotations"], 3.0)
    img = render_ref.render(p["means"], conics, p["colors"], radii, H, W,
                            opacities=torch.sigmoid(p["opacity_logits"]), normalize=normalize)
    return (img * G).sum()


def _rect_key(p):
    radii = field_ref.radii(p["log_scales"], p["rotations"], 3.0)
    return render_ref.support_rect(p["means"], radii, H, W)


@pytest.mark.parametrize("normalize", [True, False])
def test_float64_gradient_matches_central_differences(normalize):
    f = make_field(H, W, N, seed=3)
    p = {k: torch.tensor(getattr(f, k), dtype=torch.float64).requires_grad_(True) for k in NAMES}
    G = torch.tensor(np.random.default_rng(5).normal(size=(H, W, 3)), dtype=torch.float64)
    grads = torch.autograd.grad(_loss(p, G, normalize), [p[k] for k in NAMES])
    analytic = dict(zip(NAMES, grads))
    rng = np.random.default_rng(11)
    checked = 0
    worst = 0.0
    scale = max(float(g.abs().max()) for g in grads)
    with torch.no_grad():
        base = {k: v.detach().clone() for k, v in p.items()}
        rect0 = _rect_key(base)
        for k in NAMES:
            flat = base[k].view(-1)
            for idx in rng.choice(flat.numel(), size=24, replace=False):
                vals = []
                moved = False
                for sgn in (1.0, -1.0):
                    q = {kk: vv.clone() for kk, vv in base.items()}
                    q[k].view(-1)[idx] += sgn * STEP
                    if any(not torch.equal(a, b) for a, b in zip(_rect_key(q), rect0)):
                        moved = True
                        break
                    vals.append(float(_loss(q, G, normalize)))
                if moved:
                    continue  # the clipped support rectangle changed: L jumps there
                fd = (vals[0] - vals[1]) / (2 * STEP)
                an = float(analytic[k].view(-1)[idx])
                worst = max(worst, abs(fd - an) / scale)
                checked += 1
    assert checked >= 100
    assert worst <= 1e-6, worst
