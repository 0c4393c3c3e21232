"""ctypes front end of ``oracle/ss_oracle.c`` (test infrastructure only).

``load()`` builds ``oracle/_build/liboracle.so`` with gcc when it is missing.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liboracle.so"
_LIB = None

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int
_dbl = ctypes.c_double


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists() or LIB_PATH.stat().st_mtime < (HERE / "ss_oracle.c").stat().st_mtime:
        build()
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.ora_pair_count.restype = _i64
    lib.ora_pair_count.argtypes = [_f32p, _i64p, _i64, _int, _int]
    lib.ora_tile_index_offsets.restype = _i64
    lib.ora_tile_index_offsets.argtypes = [_f32p, _i64p, _i64, _int, _int, _int, _i64p]
    lib.ora_tile_index_fill.restype = None
    lib.ora_tile_index_fill.argtypes = [_f32p, _i64p, _i64, _int, _int, _int, _i64p, _i64p]
    lib.ora_render_f64.restype = None
    lib.ora_render_f64.argtypes = [_f32p, _f32p, _f32p, _i64p, ctypes.c_void_p, _i64, _int, _int,
                                   _int, _dbl, _dbl, _f64p, _f64p]
    lib.ora_backward_f64.restype = None
    lib.ora_backward_f64.argtypes = [_f64p, _f32p, _f32p, _f32p, _i64p, ctypes.c_void_p, _i64,
                                     _int, _int, _int, _dbl, _dbl, _f64p, _f64p, _f64p, _f64p,
                                     _f64p, ctypes.c_void_p]
    _LIB = lib
    return lib


def _np(x, dtype):
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(np.asarray(x), dtype=dtype)


def pair_count(means, radii, H: int, W: int) -> int:
    m, r = _np(means, np.float32), _np(radii, np.int64)
    return int(load().ora_pair_count(m, r, m.shape[0], H, W))


def tile_index(means, radii, H: int, W: int, tile_size: int):
    """(gids int64, offsets int64) with ascending ids inside each tile."""
    lib = load()
    m, r = _np(means, np.float32), _np(radii, np.int64)
    tiles = ((W + tile_size - 1) // tile_size) * ((H + tile_size - 1) // tile_size)
    offsets = np.zeros(tiles + 1, np.int64)
    total = lib.ora_tile_index_offsets(m, r, m.shape[0], H, W, tile_size, offsets)
    gids = np.zeros(max(total, 1), np.int64)
    lib.ora_tile_index_fill(m, r, m.shape[0], H, W, tile_size, offsets, gids)
    return gids[:total], offsets


def render_f64(means, conics, colors, radii, H: int, W: int, opacities=None, normalize=True,
               eps: float = 1e-8, tail: float = 0.0):
    """Float64 image (H,W,3) and raw denominator (H,W)."""
    lib = load()
    m = _np(means, np.float32)
    op = None if opacities is None else _np(opacities, np.float32)
    out = np.zeros((H, W, 3), np.float64)
    den = np.zeros((H, W), np.float64)
    lib.ora_render_f64(m, _np(conics, np.float32), _np(colors, np.float32),
                       _np(radii, np.int64), None if op is None else op.ctypes.data,
                       m.shape[0], H, W, int(bool(normalize)), float(eps), float(tail), out, den)
    return out, den


def backward_f64(grad_out, means, conics, colors, radii, H: int, W: int, opacities=None,
                 normalize=True, eps: float = 1e-8, tail: float = 0.0, den=None, out=None):
    """Float64 gradients (dict of means/conics/colors/opacities) of sum(image * grad_out)."""
    lib = load()
    if den is None or out is None:
        out, den = render_f64(means, conics, colors, radii, H, W, opacities, normalize, eps, tail)
    m = _np(means, np.float32)
    n = m.shape[0]
    op = None if opacities is None else _np(opacities, np.float32)
    g = {"means": np.zeros((n, 2)), "conics": np.zeros((n, 3)), "colors": np.zeros((n, 3)),
         "opacities": None if op is None else np.zeros(n)}
    lib.ora_backward_f64(_np(grad_out, np.float64), m, _np(conics, np.float32),
                         _np(colors, np.float32), _np(radii, np.int64),
                         None if op is None else op.ctypes.data, n, H, W, int(bool(normalize)),
                         float(eps), float(tail), _np(den, np.float64), _np(out, np.float64),
                         g["means"], g["conics"], g["colors"],
                         None if op is None else g["opacities"].ctypes.data)
    return g


def rs_render_backward_f64(grad_out, means, log_scales, rotations, colors, opacity_logits, H: int,
                           W: int, normalize=True, eps: float = 1e-8, tail: float = 0.0,
                           sigma_cutoff: float = 3.0, dilation: float = 0.0):
    """Float64 image, den and gradients of sum(image * grad_out) w.r.t. the RS field
    (means, log_scales, rotations, colors, opacity_logits) — the reference's GaussianField path
    (gaussians.py:270-321) into its renderer (render.py:180-235).

    The renderer inputs are the float32 conics, radii and opacities the field produces
    (``field_ref``, as the GPU path rounds them); the render and its gradients are evaluated in
    float64 by the C restatement, and the chain rule back to the log-scales, rotations and
    logits in float64 by torch autograd through ``field_ref.conics`` / the sigmoid.
    """
    import torch

    from . import field_ref
    ls32 = torch.as_tensor(_np(log_scales, np.float32))
    rot32 = torch.as_tensor(_np(rotations, np.float32))
    conics32 = field_ref.conics(ls32, rot32, dilation)
    radii = field_ref.radii(ls32, rot32, sigma_cutoff, dilation)
    op32 = None
    if opacity_logits is not None:
        op32 = torch.sigmoid(torch.as_tensor(_np(opacity_logits, np.float32)))
    out, den = render_f64(means, conics32, colors, radii, H, W, op32, normalize, eps, tail)
    g = backward_f64(grad_out, means, conics32, colors, radii, H, W, op32, normalize, eps, tail,
                     den=den, out=out)
    ls64 = torch.as_tensor(_np(log_scales, np.float64)).requires_grad_(True)
    rot64 = torch.as_tensor(_np(rotations, np.float64)).requires_grad_(True)
    c64 = field_ref.conics(ls64, rot64, dilation)
    g_ls, g_rot = torch.autograd.grad(c64, (ls64, rot64), torch.as_tensor(g["conics"]))
    grads = {"means": g["means"], "log_scales": g_ls.numpy(), "rotations": g_rot.numpy(),
             "colors": g["colors"], "opacity_logits": None}
    if opacity_logits is not None:
        s = 1.0 / (1.0 + np.exp(-_np(opacity_logits, np.float64)))
        grads["opacity_logits"] = g["opacities"] * s * (1.0 - s)
    return out, den, grads
