"""Host-side behaviour of the reference-mirroring Python interface (no GPU needed).

Mirrors the reference's requirement / error tests (tests/test_render.py:136-165,
tests/test_normalization_epsilon.py:32-37): CPU tensors are refused loudly (there is no CPU
fallback), bad selectors raise ValueError, and the fade / epsilon rules match render.py.
"""
from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from oracle import render_ref
from structsplat_b200 import render as R
from structsplat_b200 import render_field, render_gaussians
from structsplat_b200.structure_tensor import StructureTensorConfig, compute, gaussian_taps


def _cpu_field(n=2):
    means = torch.tensor([[3.0, 3.0], [6.0, 3.0]])[:n]
    conics = torch.tensor([[0.4, 0.0, 0.4]] * n)
    colors = torch.tensor([[1.0, 0.0, 0.0]] * n)
    radii = torch.tensor([[5, 5]] * n, dtype=torch.long)
    return means, conics, colors, radii


@pytest.mark.parametrize("mode", R.NORMALIZED_MODES + R.ADDITIVE_MODES)
def test_cpu_tensors_are_refused(mode):
    m, c, col, r = _cpu_field()
    with pytest.raises(RuntimeError, match="requires CUDA tensors"):
        render_field(m, c, col, r, 10, 10, mode=mode)


def test_rs_path_refuses_cpu():
    with pytest.raises(RuntimeError, match="requires CUDA tensors"):
        render_gaussians(torch.zeros(1, 2), torch.zeros(1, 2), torch.zeros(1), torch.zeros(1, 3),
                         4, 4)


def test_unknown_mode_and_gsplat_raise_value_error():
    m, c, col, r = _cpu_field()
    for mode in ("nope", "gsplat", "cuda_gsplat"):
        with pytest.raises(ValueError, match="unknown renderer"):
            render_field(m, c, col, r, 10, 10, mode=mode)


def test_affine_colours_are_not_silently_rendered():
    m, c, col, r = _cpu_field()
    with pytest.raises(NotImplementedError):
        render_field(m, c, col, r, 10, 10, color_grads=torch.zeros(2, 2, 3))


@pytest.mark.parametrize("value", [0.0, -1e-12, float("inf"), float("nan")])
def test_normalization_eps_validation(value):
    with pytest.raises(ValueError, match="normalization_eps must be finite and > 0"):
        R.validate_eps(value)


def test_fade_alpha_resolution_matches_reference():
    assert R.resolve_fade_alpha(False) == 0.0
    assert R.resolve_fade_alpha(True) == 1.0
    assert R.resolve_fade_alpha(True, 0.25) == 0.25
    assert R.resolve_fade_alpha(False, 3.0) == 1.0
    assert R.resolve_fade_alpha(True, -1.0) == 0.0


def test_fade_tail_is_the_float32_the_reference_subtracts():
    """render.py:106 subtracts the Python float alpha*exp(-c^2/2) from a float32 tensor."""
    q = torch.tensor([0.0, 1.0, 8.9, 9.0, 9.2, 20.0])
    for alpha in (1.0, 0.5):
        expect = render_ref.visible_weight(q, 3.0, alpha)
        tail = np.float32(R.fade_tail(3.0, alpha))
        got = torch.clamp(torch.exp(-0.5 * q) - torch.tensor(tail), min=0.0)
        assert torch.equal(got, expect)
    assert R.fade_tail(3.0, 0.0) == 0.0
    assert math.isclose(R.fade_tail(3.0, 1.0), math.exp(-4.5), rel_tol=1e-7)


def test_tile_size_validation():
    with pytest.raises(ValueError, match="tile_size"):
        R.tile_grid(8, 8, 0)
    with pytest.raises(ValueError, match="tile_size"):
        R.tile_grid(8, 8, 33)
    assert R.tile_grid(33, 29, 8) == (4, 5)


def test_gaussian_taps_match_reference_kernel():
    from oracle.structure_tensor_ref import gaussian_taps as ref_taps
    for sigma in (0.5, 1.0, 2.0, 3.0, 4.7):
        assert np.array_equal(gaussian_taps(sigma), ref_taps(sigma))


def test_structure_tensor_rejects_bad_config_and_cpu():
    with pytest.raises(ValueError, match="gradient_operator"):
        compute(np.zeros((8, 8, 3), np.float32), StructureTensorConfig(gradient_operator="x"))
    with pytest.raises(ValueError, match="color_space"):
        compute(np.zeros((8, 8, 3), np.float32), StructureTensorConfig(color_space="hsv"))
    with pytest.raises(RuntimeError, match="CUDA"):
        compute(torch.zeros(8, 8, 3))


def test_shape_validation_happens_before_launch():
    m, c, col, r = _cpu_field()
    with pytest.raises(RuntimeError, match="requires CUDA tensors"):
        R.build_tile_index(m, c, r, 8, 8, 4)


def test_codec_header_rejects_non_containers():
    import pytest as _pytest
    from structsplat_b200 import codec
    with _pytest.raises(ValueError):
        codec.blob_header(b"NOPE0" + b"\x00" * 8)
    from conftest import golden
    h = codec.blob_header(golden("codec_default_opacity.npz")["blob"].tobytes())
    assert h["n"] == 400 and h["H"] == 48 and h["W"] == 64 and h["has_opacity"]


def test_reference_extension_shim_mirrors_the_extension_checks():
    """The shim installed as the reference's _EXT raises the reference extension's RuntimeError
    messages (render_ext.cpp:94-137) before anything reaches the GPU."""
    from structsplat_b200.reference_ext import Extension
    ext = Extension()
    m, c, col, r = _cpu_field()
    op = torch.empty(0)
    gids = torch.zeros(1, dtype=torch.int32)
    offs = torch.zeros(2, dtype=torch.int32)
    with pytest.raises(RuntimeError, match="means must be a CUDA tensor"):
        ext.forward_tiled(m, c, col, r, op, gids, offs, 10, 10, True, 1e-8, 16, False, 3.0)
    with pytest.raises(RuntimeError, match="means must be a CUDA tensor"):
        ext.forward(m, c, col, r, op, 10, 10, True, 1e-8, False, 3.0)
    with pytest.raises(RuntimeError, match="must be CUDA tensors"):
        ext.build_tile_index(m, c, r, 10, 10, 16, False, 3.0)
    with pytest.raises(RuntimeError, match="means must be a CUDA tensor"):
        ext.backward(torch.zeros(10, 10, 3), m, c, col, r.int(), op, torch.zeros(10, 10),
                     torch.zeros(10, 10, 3), True, 1e-8, False, 3.0)
    for name in ("build_tile_index", "forward", "forward_tiled", "backward",
                 "backward_block_reduce", "backward_tiled"):
        assert callable(getattr(ext, name)), name
