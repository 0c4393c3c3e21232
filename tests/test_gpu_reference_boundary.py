"""The drop-in boundary, driven by the reference's own Python code.

``structsplat_b200.reference_ext.Extension`` is installed as the reference's ``cuda_render._EXT``
(the module its ``_ExactRenderCuda``, ``cuda_render.py:52-174``, calls), and the reference's
``render_cuda_exact`` / ``render_field`` run through it unchanged:

* tiled (``build_tile_index`` with its two-phase sizing → ``forward_tiled`` →
  ``backward_tiled``: the C-ABI one-call entry points) and untiled (``forward`` → ``backward`` /
  ``backward_block_reduce``, the reference's default ``mode="cuda"``), on the reference-generated
  golden cases: images within 1e-5 and gradients within 1e-4 of the reference's float32 results;
* on the 1024² / 100k-Gaussian benchmark field, against the reference's own CUDA extension
  (built unmodified for sm_100a) through the same wrapper, each error against the float64
  oracle printed;
* the ellipse-culled tile index (``ellipse_cull=True``, full fade) bit-exact against the
  reference extension's ``build_tile_index`` (``render_ext.cu:101-133,178-191``): equal offsets
  and equal per-tile sets, and the unculled index against it too.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import cuda, fwd_ok, grad_ok, rel_err, require_cuda
from oracle import c_oracle, field_ref
from ref_helpers import installed_extension, reference_extension, reference_modules
from structsplat_b200.reference_ext import Extension
from structsplat_b200.synthetic import make_field, make_stress_field, make_target

pytestmark = pytest.mark.gpu

# the reference's CUDA path has the full fade only (support_fade is a bool there)
CASES = [n for n in golden_names("render_") if float(golden(n)["fade_alpha"]) in (0.0, 1.0)]


def _leaves(z):
    op = cuda(z["opacities"]) if "opacities" in z else None
    leaves = [cuda(z["means"]), cuda(z["conics"]), cuda(z["colors"])] + (
        [op] if op is not None else [])
    for t in leaves:
        t.requires_grad_(True)
    return leaves, cuda(z["radii"]), op


def _through_wrapper(cr, z, tiled, variant="baseline", tile_size=16):
    leaves, radii, op = _leaves(z)
    img = cr.render_cuda_exact(leaves[0], leaves[1], leaves[2], radii, int(z["H"]), int(z["W"]),
                               opacities=op, normalize=bool(z["normalize"]), eps=float(z["eps"]),
                               tiled=tiled, tile_size=tile_size,
                               support_fade=float(z["fade_alpha"]) > 0,
                               sigma_cutoff=float(z["sigma_cutoff"]), backward_variant=variant)
    grads = torch.autograd.grad(img, leaves, cuda(z["grad_out"]))
    torch.cuda.synchronize()
    return img.detach(), grads


@pytest.mark.parametrize("route", ["tiled16", "tiled8", "untiled", "untiled_block_reduce"])
@pytest.mark.parametrize("name", CASES)
def test_reference_wrapper_on_the_shim_matches_reference_results(name, route):
    require_cuda()
    z = golden(name)
    with installed_extension(Extension()) as cr:
        if route.startswith("tiled"):
            img, grads = _through_wrapper(cr, z, True, tile_size=int(route[5:]))
        else:
            img, grads = _through_wrapper(
                cr, z, False, "block_reduce" if route.endswith("reduce") else "baseline")
    faded = float(z["fade_alpha"]) > 0
    e32 = rel_err(img, z["image_f32"])
    print(f"{name} {route}: fwd err vs ref f32 {e32:.2e}, vs f64 {rel_err(img, z['image_f64']):.2e}")
    assert fwd_ok(img, z["image_f32"], faded), e32
    keys = ["means", "conics", "colors"] + (["opacities"] if "opacities" in z else [])
    for key, g in zip(keys, grads):
        ok, errs = grad_ok(g, z[f"g_{key}_f32"], z[f"g_{key}_f64"])
        assert ok, (key, errs)


@pytest.mark.parametrize("mode", ["cuda", "cuda_block_reduce", "cuda_additive", "cuda_tiled",
                                  "cuda_tiled_additive"])
def test_reference_render_field_modes_run_on_the_shim(mode):
    """The reference's render_field dispatch (render.py:376-408) reaches every native call."""
    require_cuda()
    additive = mode.endswith("additive")
    z = golden("render_synthetic_64_256_additive.npz" if additive else
               "render_synthetic_64_256.npz")
    _, render = reference_modules()
    leaves, radii, op = _leaves(z)
    with installed_extension(Extension()):
        img = render.render_field(leaves[0], leaves[1], leaves[2], radii, int(z["H"]),
                                  int(z["W"]), mode=mode, opacities=op,
                                  normalization_eps=float(z["eps"]))
        grads = torch.autograd.grad(img, leaves, cuda(z["grad_out"]))
    assert fwd_ok(img.detach(), z["image_f32"], False)
    keys = ["means", "conics", "colors"] + (["opacities"] if op is not None else [])
    for key, g in zip(keys, grads):
        assert grad_ok(g, z[f"g_{key}_f32"], z[f"g_{key}_f64"])[0], key


def _c2_inputs():
    H = W = 1024
    f = make_field(H, W, 100_000, seed=0)
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    host = {"means": f.means, "conics": field_ref.conics(ls, rot).numpy(),
            "colors": f.colors, "radii": field_ref.radii(ls, rot, 3.0).numpy(),
            "opacities": torch.sigmoid(torch.tensor(f.opacity_logits)).numpy(),
            "grad_out": make_target(H, W, seed=1) - np.float32(0.5)}
    return H, W, host


@pytest.mark.parametrize("normalize", [True, False])
def test_benchmark_field_shim_matches_reference_extension(normalize):
    """1024² / 100k Gaussians (the benchmark field): the reference wrapper on the shim against
    the reference wrapper on its own extension (tiled arm, 16-px tiles), both against float64."""
    require_cuda()
    ref_ext = reference_extension()
    H, W, host = _c2_inputs()
    z = {"H": H, "W": W, "normalize": normalize, "eps": 1e-8, "fade_alpha": 0.0,
         "sigma_cutoff": 3.0, **host}
    results = {}
    for label, ext in (("ours", Extension()), ("reference", ref_ext)):
        with installed_extension(ext) as cr:
            results[label] = _through_wrapper(cr, z, True)
    out64, den64 = c_oracle.render_f64(host["means"], host["conics"], host["colors"],
                                       host["radii"], H, W, host["opacities"], normalize)
    g64 = c_oracle.backward_f64(host["grad_out"], host["means"], host["conics"], host["colors"],
                                host["radii"], H, W, host["opacities"], normalize,
                                den=den64, out=out64)
    img, grads = results["ours"]
    ref_img, ref_grads = results["reference"]
    e_ref, e64, ref64 = rel_err(img, ref_img), rel_err(img, out64), rel_err(ref_img, out64)
    print(f"C2 normalize={normalize}: fwd err vs ref ext {e_ref:.2e}, vs f64 {e64:.2e} "
          f"(ref ext vs f64 {ref64:.2e})")
    assert e_ref <= 1e-5
    for key, g, rg in zip(("means", "conics", "colors", "opacities"), grads, ref_grads):
        ok, (e32, e, own) = grad_ok(g, rg, g64[key])
        print(f"  {key}: grad err vs ref ext {e32:.2e}, vs f64 {e:.2e} (ref ext vs f64 {own:.2e})")
        assert ok, key


def _sets_equal(gids_a, off_a, gids_b, off_b) -> bool:
    if not np.array_equal(off_a, off_b):
        return False
    for t in range(len(off_a) - 1):
        a = np.sort(gids_a[off_a[t]:off_a[t + 1]])
        b = np.sort(gids_b[off_b[t]:off_b[t + 1]])
        if not np.array_equal(a, b):
            return False
    return True


def _index_fields():
    """(name, H, W, means, conics, radii) cases for the index comparison."""
    out = []
    z = golden("render_elongated_fade.npz")
    out.append(("elongated_fade", int(z["H"]), int(z["W"]), z["means"], z["conics"], z["radii"]))
    rng = np.random.default_rng(22)
    N, H, W = 400, 96, 100
    means = np.stack([rng.uniform(-3, W + 3, N), rng.uniform(-3, H + 3, N)], 1).astype(np.float32)
    ls = np.log(np.stack([np.exp(rng.uniform(np.log(2), np.log(12), N)),
                          np.exp(rng.uniform(np.log(0.5), np.log(1.2), N))], 1)).astype(np.float32)
    rot = rng.uniform(0, np.pi, N).astype(np.float32)
    out.append(("thin_rotated", H, W, means,
                field_ref.conics(torch.tensor(ls), torch.tensor(rot)).numpy(),
                field_ref.radii(torch.tensor(ls), torch.tensor(rot), 3.0).numpy()))
    H = W = 256
    angle = np.random.default_rng(3).uniform(0, np.pi, (H, W)).astype(np.float32)
    f = make_stress_field(H, W, 15_000, seed=4, along_edge_angle=angle)
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    out.append(("stress_256", H, W, f.means, field_ref.conics(ls, rot).numpy(),
                field_ref.radii(ls, rot, 3.0).numpy()))
    H, W, host = _c2_inputs()
    out.append(("benchmark_1024", H, W, host["means"], host["conics"], host["radii"]))
    return out


INDEX_FIELDS = None


def _fields():
    global INDEX_FIELDS
    if INDEX_FIELDS is None:
        INDEX_FIELDS = _index_fields()
    return INDEX_FIELDS


@pytest.mark.parametrize("cutoff", [2.0, 3.0])
@pytest.mark.parametrize("tile_size", [8, 16, 32])
@pytest.mark.parametrize("cull", [True, False])
@pytest.mark.parametrize("case", range(4))
def test_tile_index_bit_exact_against_reference_extension(case, cull, tile_size, cutoff):
    require_cuda()
    ref_ext = reference_extension()
    name, H, W, means, conics, radii = _fields()[case]
    if cutoff != 3.0:  # radii follow the cutoff: scale the 3σ half-widths
        radii = np.maximum(np.ceil(radii * (cutoff / 3.0)).astype(np.int64), 1)
    m, c, r = cuda(means, torch.float32), cuda(conics, torch.float32), cuda(radii, torch.int64)
    ours = Extension().build_tile_index(m, c, r, H, W, tile_size, cull, cutoff)
    ref = ref_ext.build_tile_index(m, c, r, H, W, tile_size, cull, cutoff)
    torch.cuda.synchronize()
    og, oo = (t.cpu().numpy().astype(np.int64) for t in ours)
    rg, ro = (t.cpu().numpy().astype(np.int64) for t in ref)
    kept = int(ro[-1])
    print(f"{name} ts={tile_size} cull={cull} cutoff={cutoff}: {kept} entries "
          f"(reference pairs before the cull: {rg.size})")
    assert og.size == kept
    assert _sets_equal(og, oo, rg[:kept], ro), name
    # the library lists each tile in ascending id, which is the reference's stable order too
    assert np.array_equal(og, rg[:kept])
    if cull and name == "stress_256":
        assert kept < rg.size  # the elongated Gaussians' rectangles hold culled tiles
