"""The oracle's activity and raw weight map reproduce the reference's (fixtures pass_*)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from oracle import field_ref, render_ref

CASES = golden_names("pass_")


@pytest.mark.parametrize("name", CASES)
def test_activity_matches_reference(name):
    z = golden(name)
    got = render_ref.activity(torch.tensor(z["means"]), torch.tensor(z["conics"]),
                              torch.tensor(z["radii"]), int(z["H"]), int(z["W"]),
                              fade_alpha=float(z["fade_alpha"]))
    assert np.allclose(got.numpy(), z["activity"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("name", CASES)
def test_raw_weight_map_matches_reference(name):
    z = golden(name)
    H, W = int(z["H"]), int(z["W"])
    p = {k: torch.tensor(z[k]).requires_grad_(True)
         for k in ("means", "log_scales", "rotations", "opacity_logits")}
    conics = field_ref.conics(p["log_scales"], p["rotations"])
    radii = field_ref.radii(p["log_scales"], p["rotations"], 3.0)
    _, den = render_ref.render(p["means"], conics, conics, radii, H, W,
                               opacities=torch.sigmoid(p["opacity_logits"]), normalize=False,
                               fade_alpha=float(z["fade_alpha"]), return_den=True)
    den = den.reshape(-1)
    assert np.allclose(den.detach().numpy(), z["den"], rtol=1e-5, atol=1e-7)
    grads = torch.autograd.grad((den * torch.tensor(z["G"])).sum(), list(p.values()))
    for k, g in zip(p, grads):
        ref = z[f"g_{k}"]
        assert np.abs(g.numpy() - ref).max() <= 1e-4 * max(np.abs(ref).max(), 1e-12), k
