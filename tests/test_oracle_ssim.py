"""The SSIM oracle against the reference's own metrics.ssim (tests/golden/ssim_*.npz): value,
gradient w.r.t. the rendered image, and the fit loop's L1 + SSIM mix."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import ssim_ref

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLDEN.glob("ssim_*.npz"))


def test_fixtures_present():
    assert len(CASES) >= 3


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_ssim(name):
    z = np.load(GOLDEN / f"{name}.npz")
    pred = torch.tensor(z["pred"], requires_grad=True)
    target = torch.tensor(z["target"])
    s = ssim_ref.ssim(pred, target)
    (g,) = torch.autograd.grad(s, pred)
    assert abs(float(s.detach()) - float(z["ssim"])) <= 1e-6
    assert abs(float(z["ssim_cached"]) - float(z["ssim"])) <= 1e-6
    scale = np.abs(z["grad_ssim"]).max()
    assert np.abs(g.numpy() - z["grad_ssim"]).max() <= 1e-5 * scale


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_mixed_loss(name):
    z = np.load(GOLDEN / f"{name}.npz")
    pred = torch.tensor(z["pred"], requires_grad=True)
    loss = ssim_ref.mixed_loss(pred, torch.tensor(z["target"]), float(z["weight"]), "l1")
    (g,) = torch.autograd.grad(loss, pred)
    assert abs(float(loss.detach()) - float(z["loss"])) <= 1e-6
    scale = np.abs(z["grad_loss"]).max()
    assert np.abs(g.numpy() - z["grad_loss"]).max() <= 1e-5 * scale
