"""Forward and backward parity of the B200 renderer against the reference's own results.

Golden vectors come from the reference's ``render_field`` (tests/golden).  Bars: forward images
within 1e-5 relative and gradients within 1e-4 relative (norm-wise: max |got − ref| / max |ref|)
of the reference's float32 results; each case also states its error against the reference
evaluated in float64.  Where the reference's own float32 gradient is itself far from float64
(a gradient made of cancelling terms, e.g. a lone or single-colour splat whose
dw = dnum·c + dden is rounding noise), matching it is meaningless; there the bar is to be no
less accurate than it: error vs float64 ≤ max(1e-4, 2 × the reference's own float32 error).  Cases with the full support fade are ill-conditioned at the cutoff
(exp(−q/2) − exp(−c²/2) cancels): for those the forward is compared element-wise with a floor
and the float64 yardstick shows the reference float32 path has the same conditioning.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import GRAD_TOL, cuda, fwd_ok, grad_ok, rel_err, require_cuda
from structsplat_b200 import render_b200, render_gaussians
from structsplat_b200 import render as R

pytestmark = pytest.mark.gpu

RENDER_CASES = golden_names("render_")


def _case(z):
    op = cuda(z["opacities"]) if "opacities" in z.files else None
    return (cuda(z["means"]), cuda(z["conics"]), cuda(z["colors"]), cuda(z["radii"]), op)


def _render(z, deterministic=False, want_grads=True):
    m, c, col, r, op = _case(z)
    leaves = [m, c, col] + ([op] if op is not None else [])
    for t in leaves:
        t.requires_grad_(want_grads)
    alpha = float(z["fade_alpha"])
    img = render_b200(m, c, col, r, int(z["H"]), int(z["W"]), opacities=op,
                      normalize=bool(z["normalize"]), eps=float(z["eps"]),
                      support_fade=alpha > 0, support_fade_alpha=alpha,
                      sigma_cutoff=float(z["sigma_cutoff"]), deterministic=deterministic)
    if not want_grads:
        return img.detach(), None
    grads = torch.autograd.grad(img, leaves, cuda(z["grad_out"]))
    torch.cuda.synchronize()
    return img.detach(), grads


def _grad_ok(got, z, key, prefix="g"):
    return grad_ok(got, z[f"{prefix}_{key}_f32"], z[f"{prefix}_{key}_f64"])


def _fwd_error_ok(img, z):
    return fwd_ok(img, z["image_f32"], float(z["fade_alpha"]) > 0)


@pytest.mark.parametrize("name", RENDER_CASES)
def test_forward_matches_reference(name):
    require_cuda()
    z = golden(name)
    img, _ = _render(z, want_grads=False)
    e32, e64 = rel_err(img, z["image_f32"]), rel_err(img, z["image_f64"])
    ref64 = rel_err(z["image_f32"], z["image_f64"])
    print(f"{name}: fwd err vs ref f32 {e32:.2e}, vs f64 {e64:.2e} (ref f32 vs f64 {ref64:.2e})")
    assert _fwd_error_ok(img, z), (e32, e64)


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("name", RENDER_CASES)
def test_gradients_match_reference(name, deterministic):
    require_cuda()
    z = golden(name)
    _, grads = _render(z, deterministic=deterministic)
    keys = ["means", "conics", "colors"] + (["opacities"] if "opacities" in z.files else [])
    for key, g in zip(keys, grads):
        ok, (e32, e64, ref_err) = _grad_ok(g, z, key)
        print(f"{name} {key}: grad err vs ref f32 {e32:.2e}, vs f64 {e64:.2e} "
              f"(ref f32 vs f64 {ref_err:.2e})")
        assert ok, (key, e32, e64, ref_err)


@pytest.mark.parametrize("name", RENDER_CASES)
def test_rs_field_path_matches_reference(name):
    """render_gaussians (fused projection + chain rule) against autograd through the
    reference's GaussianField.conics / radii / opacity_values."""
    require_cuda()
    z = golden(name)
    m, ls, rot, col = (cuda(z[k]) for k in ("means", "log_scales", "rotations", "colors"))
    logits = cuda(z["opacity_logits"]) if "opacity_logits" in z.files else None
    leaves = [m, ls, rot, col] + ([logits] if logits is not None else [])
    for t in leaves:
        t.requires_grad_(True)
    alpha = float(z["fade_alpha"])
    img = render_gaussians(m, ls, rot, col, int(z["H"]), int(z["W"]), opacity_logits=logits,
                           normalize=bool(z["normalize"]), eps=float(z["eps"]),
                           sigma_cutoff=float(z["sigma_cutoff"]), dilation=float(z["dilation"]),
                           support_fade=alpha > 0, support_fade_alpha=alpha)
    grads = torch.autograd.grad(img, leaves, cuda(z["grad_out"]))
    assert _fwd_error_ok(img.detach(), z)
    keys = ["means", "log_scales", "rotations", "colors"] + (
        ["opacity_logits"] if logits is not None else [])
    for key, g in zip(keys, grads):
        ok, (e32, e64, ref_err) = _grad_ok(g, z, key, prefix="rs")
        print(f"{name} rs {key}: grad err vs ref f32 {e32:.2e}, vs f64 {e64:.2e} "
              f"(ref f32 vs f64 {ref_err:.2e})")
        assert ok, (key, e32, e64, ref_err)


def test_rs_projection_matches_reference_conics_and_radii():
    require_cuda()
    from structsplat_b200.field import project
    for name in RENDER_CASES:
        z = golden(name)
        logits = cuda(z["opacity_logits"]) if "opacity_logits" in z.files else None
        _, conics, radii = project(cuda(z["means"]), cuda(z["log_scales"]), cuda(z["rotations"]),
                                   cuda(z["colors"]), logits, int(z["H"]), int(z["W"]),
                                   float(z["sigma_cutoff"]), float(z["dilation"]),
                                   want_conics=True)
        assert np.array_equal(radii.cpu().numpy(), z["radii"]), name
        assert rel_err(conics, z["conics"]) <= 1e-6, name


def test_deterministic_backward_is_bitwise_reproducible():
    require_cuda()
    z = golden("render_synthetic_64_256.npz")
    _, g1 = _render(z, deterministic=True)
    _, g2 = _render(z, deterministic=True)
    for a, b in zip(g1, g2):
        assert torch.equal(a, b)


def test_forward_is_bitwise_reproducible():
    require_cuda()
    z = golden("render_synthetic_64_256.npz")
    a, _ = _render(z, want_grads=False)
    b, _ = _render(z, want_grads=False)
    assert torch.equal(a, b)


def test_truncated_index_renders_identically():
    """With too small a capacity the affected tiles scan every Gaussian in ascending id: the
    image is bitwise identical and the status word reports the overflow."""
    require_cuda()
    z = golden("render_synthetic_64_256.npz")
    m, c, col, r, op = _case(z)
    H, W = int(z["H"]), int(z["W"])
    rec = R.pack_records(m, c, col, r, op, H, W)
    full = R.index_from_records(rec, m.shape[0], H, W, exact=True)
    part = R.index_from_records(rec, m.shape[0], H, W, capacity=full.capacity // 3)
    out_f, den_f = R._forward(rec, m.shape[0], full, H, W, True, 1e-8, 0.0, m.device)
    out_p, den_p = R._forward(rec, m.shape[0], part, H, W, True, 1e-8, 0.0, m.device)
    torch.cuda.synchronize()
    assert int(full.status.item()) == 0
    assert int(part.status.item()) & 1
    assert torch.equal(out_f, out_p) and torch.equal(den_f, den_p)
    go = cuda(z["grad_out"])
    g_f = R._backward(go, rec, m.shape[0], den_f, out_f, full, H, W, True, 1e-8, 0.0, True,
                      False, m.device)
    g_p = R._backward(go, rec, m.shape[0], den_p, out_p, part, H, W, True, 1e-8, 0.0, True,
                      False, m.device)
    for a, b in zip(g_f, g_p):
        assert rel_err(b, a) <= 1e-6


def test_empty_field_renders_zeros():
    require_cuda()
    e = torch.zeros(0, 2, device="cuda")
    img = render_b200(e, torch.zeros(0, 3, device="cuda"), torch.zeros(0, 3, device="cuda"),
                      torch.zeros(0, 2, dtype=torch.long, device="cuda"), 8, 9)
    assert img.shape == (8, 9, 3) and torch.count_nonzero(img) == 0


def test_nonfinite_means_are_dropped():
    """render_ext.cu:25-34 semantics: NaN / inf / huge centres contribute nothing."""
    require_cuda()
    means = cuda(np.array([[5.0, 5.0], [np.nan, 3.0], [1e12, 1e12], [np.inf, 2.0]], np.float32))
    conics = cuda(np.tile(np.array([[0.44, 0.0, 0.44]], np.float32), (4, 1)))
    colors = torch.ones(4, 3, device="cuda")
    radii = torch.full((4, 2), 5, dtype=torch.long, device="cuda")
    img = render_b200(means, conics, colors, radii, 12, 12)
    one = render_b200(means[:1], conics[:1], colors[:1], radii[:1], 12, 12)
    assert torch.isfinite(img).all() and torch.equal(img, one)


@pytest.mark.parametrize("normalize", [True, False])
def test_infinite_colour_on_a_large_rectangle_gives_the_reference_nans(normalize):
    """An elongated Gaussian (rectangle > 48 px) with an infinite colour channel: where its
    weight underflows to 0 the reference's product 0 * inf is NaN, so the block skip for
    underflowed weights must not drop it.  NaN pattern and finite values as the oracle."""
    require_cuda()
    from oracle import render_ref
    H = W = 96
    ang = np.float32(np.pi / 4)
    sx, sy = np.float32(30.0), np.float32(1.2)  # standard deviations along / across
    c, s = np.cos(ang), np.sin(ang)
    cov = np.array([[c * c * sx * sx + s * s * sy * sy, c * s * (sx * sx - sy * sy)],
                    [c * s * (sx * sx - sy * sy), s * s * sx * sx + c * c * sy * sy]])
    inv = np.linalg.inv(cov)
    conic = np.array([[inv[0, 0], inv[0, 1], inv[1, 1]]], np.float32)
    rad = np.ceil(3.0 * np.sqrt(np.diag(cov))).astype(np.int64)[None, :]
    means = np.array([[48.3, 47.6]], np.float32)
    colors = np.array([[np.inf, 0.5, 0.25]], np.float32)
    img = render_b200(cuda(means), cuda(conic), cuda(colors), cuda(rad), H, W,
                      normalize=normalize).cpu()
    ref = render_ref.render(torch.tensor(means), torch.tensor(conic), torch.tensor(colors),
                            torch.tensor(rad), H, W, normalize=normalize)
    assert int(rad.max()) > 24  # a rectangle wider than 48 px
    nan_ref, nan_img = torch.isnan(ref), torch.isnan(img)
    assert nan_ref.sum() > 1000
    assert not (nan_ref & ~nan_img).any()  # every NaN of the reference
    # the only other NaNs: pixels whose reference weight is subnormal (inf there), which the
    # flush-to-zero exponential returns as 0 (0 * inf)
    extra = nan_img & ~nan_ref
    assert torch.isinf(ref[extra]).all() and extra.sum() <= 0.1 * nan_ref.sum()
    fin = torch.isfinite(ref) & torch.isfinite(img)
    assert torch.equal(fin, torch.isfinite(ref))  # the finite channels stay finite
    # along the major axis the conic's terms (~150 each 30 px out) cancel to q ~ 1, so both
    # float32 evaluations carry ~1e-5 relative error in the weight there
    assert rel_err(img[fin], ref[fin]) <= 1e-4


def test_zero_sized_image():
    require_cuda()
    m = torch.tensor([[1.0, 1.0]], device="cuda")
    img = render_b200(m, torch.ones(1, 3, device="cuda"), torch.ones(1, 3, device="cuda"),
                      torch.ones(1, 2, dtype=torch.long, device="cuda"), 0, 5)
    assert img.shape == (0, 5, 3)


@pytest.mark.parametrize("name", ["render_synthetic_64_256.npz", "render_elongated_fade.npz",
                                  "render_matrix_add_op_d3_f1.npz"])
def test_render_tile_sizes_agree(name):
    """16x16 and 32x32 render tiles give every 8x8 block the same hits in the same order, so the
    images are identical.  With the full support fade the ellipse cull drops each tile's
    zero-weight pairs, which differ between the tile sizes: a block may then list a Gaussian
    that contributes exact zeros in one tiling and not in the other, which moves the later hits
    to other partial sums; those images agree to float rounding.  Gradients agree to rounding."""
    require_cuda()
    z = golden(name)
    outs = []
    for ts in (16, 32):
        m, c, col, r, op = _case(z)
        leaves = [m, c, col] + ([op] if op is not None else [])
        for t in leaves:
            t.requires_grad_(True)
        alpha = float(z["fade_alpha"])
        img = render_b200(m, c, col, r, int(z["H"]), int(z["W"]), opacities=op,
                          normalize=bool(z["normalize"]), eps=float(z["eps"]),
                          support_fade=alpha > 0, support_fade_alpha=alpha, tile_size=ts)
        outs.append((img.detach(), torch.autograd.grad(img, leaves, cuda(z["grad_out"]))))
    if float(z["fade_alpha"]) >= 1.0:
        assert rel_err(outs[0][0], outs[1][0]) <= 1e-6
    else:
        assert torch.equal(outs[0][0], outs[1][0])
    for a, b in zip(outs[0][1], outs[1][1]):
        assert rel_err(a, b) <= 1e-5


@pytest.mark.parametrize("normalize", [True, False])
def test_gpu_gradients_on_the_finite_difference_case(normalize):
    """GPU RS-parameter gradients vs the float64 gradient that tests/test_fd_gradients.py pins
    to central differences (64x64, 256 Gaussians, step 1e-4)."""
    require_cuda()
    from oracle import field_ref, render_ref
    from structsplat_b200.synthetic import make_field
    names = ("means", "log_scales", "rotations", "colors", "opacity_logits")
    f = make_field(64, 64, 256, seed=3)
    G = np.random.default_rng(5).normal(size=(64, 64, 3))
    p64 = {k: torch.tensor(getattr(f, k), dtype=torch.float64).requires_grad_(True) for k in names}
    img64 = render_ref.render(p64["means"], field_ref.conics(p64["log_scales"], p64["rotations"]),
                              p64["colors"], field_ref.radii(p64["log_scales"], p64["rotations"], 3.0),
                              64, 64, opacities=torch.sigmoid(p64["opacity_logits"]),
                              normalize=normalize)
    g64 = torch.autograd.grad((img64 * torch.tensor(G)).sum(), [p64[k] for k in names])
    leaves = [torch.tensor(getattr(f, k), device="cuda").requires_grad_(True) for k in names]
    img = render_gaussians(*leaves[:4], 64, 64, opacity_logits=leaves[4], normalize=normalize)
    g32 = torch.autograd.grad(img, leaves, torch.tensor(G, dtype=torch.float32, device="cuda"))
    for k, a, b in zip(names, g32, g64):
        err = rel_err(a, b)
        print(f"{k}: rel err vs float64 {err:.2e}")
        assert err <= GRAD_TOL, k
