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


@pytest.mark.parametrize("H, W, grad_sigma, tensor_sigma, op, space", [
    (70, 97, 1.0, 2.0, "central", "luma"),    # tiles cut by both image edges
    (129, 33, 1.0, 3.0, "sobel", "rgb"),      # the stress workload's tensor blur
    (64, 80, 4.5, 2.0, "scharr", "luma"),     # a gradient blur wider than the tiles' halo
    (40, 52, 0.0, 4.5, "central", "rgb"),     # no gradient blur, a wide tensor blur
])
def test_tile_and_per_pass_kernels_match_the_oracle(H, W, grad_sigma, tensor_sigma, op, space):
    """The shared-memory tile kernels (blur radii up to 12) and the per-pass kernels (wider
    blurs) against the CPU oracle's restatement of structure_tensor.compute on ragged images:
    the maps to float32 rounding, the float64 statistics from the exact order statistics."""
    require_cuda()
    from oracle import structure_tensor_ref as ref
    from structsplat_b200.synthetic import make_target
    img = make_target(H, W, seed=H + W)
    cfg = StructureTensorConfig(grad_sigma, tensor_sigma, op, space)
    t = compute(img, cfg)
    want = ref.compute(img, ref.TensorConfig(grad_sigma=grad_sigma, tensor_sigma=tensor_sigma,
                                             gradient_operator=op, color_space=space))
    scale = max(float(np.abs(want.energy).max()), 1e-30)
    for attr in ("lam1", "lam2", "energy"):
        err = np.abs(getattr(t, attr).cpu().numpy() - getattr(want, attr)).max() / scale
        assert err <= 1e-6, (attr, err)
    assert abs(t.energy_ref - float(want.energy_ref)) <= 1e-6 * float(want.energy_ref)
    assert (t.label.cpu().numpy() != want.label).mean() <= 1e-3
