"""Pins the CPU oracle to golden vectors produced by the reference implementation itself.

The fixtures in tests/golden were generated by tests/golden/make_golden.py from the reference's
own ``render_field`` (float32 and float64), ``GaussianField``, ``_build_tile_index`` and
``structure_tensor.compute``.  These tests need no GPU.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from oracle import c_oracle, field_ref, render_ref, tile_index_ref
from oracle import structure_tensor_ref as st_ref

RENDER_CASES = golden_names("render_")
TILE_CASES = golden_names("tile_")
ST_CASES = golden_names("st_")


def _inputs(z):
    op = torch.tensor(z["opacities"]) if "opacities" in z.files else None
    return (torch.tensor(z["means"]), torch.tensor(z["conics"]), torch.tensor(z["colors"]),
            torch.tensor(z["radii"]), op)


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)) if b.size else 0.0


def test_fixture_inventory():
    assert len(RENDER_CASES) >= 20 and len(TILE_CASES) >= 5 and len(ST_CASES) >= 8


@pytest.mark.parametrize("name", RENDER_CASES)
def test_torch_oracle_reproduces_reference_render(name):
    z = golden(name)
    m, c, col, r, op = _inputs(z)
    img, _, g = render_ref.render_with_grads(
        m, c, col, r, int(z["H"]), int(z["W"]), torch.tensor(z["grad_out"]), op,
        bool(z["normalize"]), float(z["eps"]), float(z["sigma_cutoff"]), float(z["fade_alpha"]))
    assert _rel(img, z["image_f32"]) <= 1e-6
    # float32 sums of ~1,000 terms per pixel (the streamed cases) depend on the summation order,
    # which the oracle's single pass and the reference's chunked index_add do not share
    gtol = 1e-5 if "streamed" in name else 2e-6
    for key in ("means", "conics", "colors"):
        assert _rel(g[key], z[f"g_{key}_f32"]) <= gtol, key
    if op is not None:
        assert _rel(g["opacities"], z["g_opacities_f32"]) <= gtol


@pytest.mark.parametrize("name", RENDER_CASES)
def test_field_oracle_reproduces_reference_projection(name):
    z = golden(name)
    ls, rot = torch.tensor(z["log_scales"]), torch.tensor(z["rotations"])
    d = float(z["dilation"])
    assert np.array_equal(field_ref.conics(ls, rot, d).numpy(), z["conics"])
    assert np.array_equal(field_ref.radii(ls, rot, float(z["sigma_cutoff"]), d).numpy(),
                          z["radii"])
    if "opacity_logits" in z.files:
        assert np.array_equal(field_ref.opacity_values(torch.tensor(z["opacity_logits"])).numpy(),
                              z["opacities"])


@pytest.mark.parametrize("name", RENDER_CASES)
def test_c_float64_oracle_matches_torch_float64(name):
    """The C float64 forward/backward equals the reference equations evaluated in float64 on the
    same (float32) inputs."""
    z = golden(name)
    m, c, col, r, op = _inputs(z)
    H, W = int(z["H"]), int(z["W"])
    alpha, cut, eps = float(z["fade_alpha"]), float(z["sigma_cutoff"]), float(z["eps"])
    norm = bool(z["normalize"])
    tail = render_ref.fade_tail(cut, alpha)
    img64, den64, g64 = render_ref.render_with_grads(
        m.double(), c.double(), col.double(), r, H, W, torch.tensor(z["grad_out"]).double(),
        None if op is None else op.double(), norm, eps, cut, alpha)
    out, den = c_oracle.render_f64(m, c, col, r, H, W, op, norm, eps, tail)
    assert _rel(out, img64) <= 1e-12
    assert _rel(den, den64) <= 1e-12
    g = c_oracle.backward_f64(z["grad_out"], m, c, col, r, H, W, op, norm, eps, tail)
    for key in ("means", "conics", "colors") + (("opacities",) if op is not None else ()):
        assert _rel(g[key], g64[key]) <= 1e-8, key  # cancellation-heavy sums differ in order


@pytest.mark.parametrize("name", TILE_CASES)
def test_tile_index_oracles_match_reference(name):
    z = golden(name)
    H, W, ts = int(z["H"]), int(z["W"]), int(z["tile_size"])
    gids, offsets = tile_index_ref.build_tile_index(torch.tensor(z["means"]),
                                                    torch.tensor(z["radii"]), H, W, ts)
    assert np.array_equal(offsets, z["offsets"])
    assert np.array_equal(gids, z["gids_sorted"])
    cg, coff = c_oracle.tile_index(z["means"], z["radii"], H, W, ts)
    assert np.array_equal(coff, z["offsets"])
    assert np.array_equal(cg, z["gids_sorted"])


def test_tile_index_known_answer():
    """tests/test_render.py:167-172 of the reference."""
    gids, offsets = tile_index_ref.build_tile_index(
        torch.tensor([[2.0, 2.0], [20.0, 20.0]]), torch.tensor([[1, 1], [1, 1]]), 8, 8, 4)
    assert offsets.tolist() == [0, 1, 1, 1, 1]
    assert gids.tolist() == [0]


def test_nonfinite_centre_has_empty_support():
    m = np.array([[5.0, 5.0], [np.nan, 3.0], [np.inf, 1.0], [2.0, -np.inf]], np.float32)
    r = np.full((4, 2), 2, np.int64)
    gids, off = c_oracle.tile_index(m, r, 12, 12, 4)
    assert 1 not in gids and 2 not in gids and 3 not in gids
    assert c_oracle.pair_count(m, r, 12, 12) == 25


@pytest.mark.parametrize("name", ST_CASES)
def test_structure_tensor_oracle_matches_reference(name):
    z = golden(name)
    cfg = st_ref.TensorConfig(float(z["grad_sigma"]), float(z["tensor_sigma"]),
                              str(z["gradient_operator"]), str(z["color_space"]),
                              float(z["flat_frac"]), float(z["corner_frac"]))
    t = st_ref.compute(z["img"], cfg)
    for a, b in (("lam1", "lam1"), ("lam2", "lam2"), ("across_edge_angle", "angle"),
                 ("coherence", "coherence"), ("energy", "energy")):
        assert np.array_equal(getattr(t, a), z[b]), a
    assert np.array_equal(t.label, z["label"])
    assert t.energy_ref == float(z["energy_ref"])


def test_pair_count_matches_rect_areas():
    from structsplat_b200.synthetic import make_field
    f = make_field(64, 80, 500, seed=1)
    r = field_ref.radii(torch.tensor(f.log_scales), torch.tensor(f.rotations), 3.0)
    expect = render_ref.pair_count(torch.tensor(f.means), r, 64, 80)
    assert c_oracle.pair_count(f.means, r, 64, 80) == expect > 0
