"""GPU structure tensor against the reference's ``structure_tensor.compute`` (golden vectors).

Blurs, gradients and products follow NumPy's float32 operation order, so lam1 / lam2 / energy
/ coherence agree to a few float32 ulps; the angle goes through atan2f, whose last-bit rounding
differs from NumPy's, and is compared where the structure is not degenerate.  Labels compare
thresholds computed from the same float64 statistics.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, golden_names
from gpu_helpers import require_cuda
from structsplat_b200.structure_tensor import StructureTensorConfig, compute

pytestmark = pytest.mark.gpu


def _cfg(z):
    return StructureTensorConfig(float(z["grad_sigma"]), float(z["tensor_sigma"]),
                                 str(z["gradient_operator"]), str(z["color_space"]),
                                 float(z["flat_frac"]), float(z["corner_frac"]))


@pytest.mark.parametrize("name", golden_names("st_"))
def test_structure_tensor_matches_reference(name):
    require_cuda()
    z = golden(name)
    t = compute(z["img"], _cfg(z))
    scale = max(float(np.abs(z["energy"]).max()), 1e-30)
    for attr, key in (("lam1", "lam1"), ("lam2", "lam2"), ("energy", "energy")):
        got = getattr(t, attr).cpu().numpy()
        err = np.abs(got - z[key]).max() / scale
        print(f"{name} {attr}: max err / max energy {err:.2e}")
        assert err <= 1e-6, attr
    strong = z["energy"] > 1e-3 * scale
    coh = t.coherence.cpu().numpy()
    assert np.abs(coh - z["coherence"])[strong].max(initial=0.0) <= 1e-5
    ang = t.across_edge_angle.cpu().numpy()
    d = np.abs(np.angle(np.exp(2j * (ang - z["angle"])))) / 2
    assert d[strong & (z["coherence"] > 1e-3)].max(initial=0.0) <= 1e-4
    assert abs(t.energy_ref - float(z["energy_ref"])) <= 1e-6 * float(z["energy_ref"])
    mismatch = (t.label.cpu().numpy() != z["label"]).mean()
    assert mismatch <= 1e-3, mismatch


def test_torch_input_and_rgb_channels():
    require_cuda()
    import torch
    z = golden("st_isoluminant_rgb.npz")
    img = torch.as_tensor(z["img"]).cuda()
    t_rgb = compute(img, StructureTensorConfig(color_space="rgb"))
    t_luma = compute(img, StructureTensorConfig(color_space="luma"))
    assert float(t_rgb.energy.max()) > 50 * (float(t_luma.energy.max()) + 1e-9)
