"""Shared helpers of the GPU parity tests."""
from __future__ import annotations

import numpy as np
import pytest
import torch


def require_cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")


def rel_err(got, ref) -> float:
    """max |got − ref| / max |ref| (norm-wise relative error)."""
    got = np.asarray(got.detach().cpu() if torch.is_tensor(got) else got, np.float64)
    ref = np.asarray(ref.detach().cpu() if torch.is_tensor(ref) else ref, np.float64)
    if ref.size == 0:
        return 0.0
    return float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30))


def elementwise_rel(got, ref, floor: float) -> float:
    """max over elements of |got − ref| / max(|ref|, floor)."""
    got = np.asarray(got.detach().cpu() if torch.is_tensor(got) else got, np.float64)
    ref = np.asarray(ref.detach().cpu() if torch.is_tensor(ref) else ref, np.float64)
    if ref.size == 0:
        return 0.0
    return float((np.abs(got - ref) / np.maximum(np.abs(ref), floor)).max())


def cuda(x, dtype=None):
    t = torch.as_tensor(np.asarray(x))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


FWD_TOL = 1e-5   # forward images: relative to the reference's float32 result
GRAD_TOL = 1e-4  # gradients: relative to the reference's float32 result


def grad_ok(got, ref32, ref64):
    """Gradient bar against the reference's float32 gradient ``ref32``; where that gradient is
    itself far from float64 (cancelling terms), the bar is to be no less accurate than it:
    error vs float64 ≤ max(GRAD_TOL, 2 × the reference's own float32 error).
    Returns (ok, (err vs ref32, err vs f64, ref32's own error))."""
    e32 = rel_err(got, ref32)
    e64 = rel_err(got, ref64)
    ref_err = rel_err(ref32, ref64)
    if ref_err <= GRAD_TOL / 10:
        return e32 <= GRAD_TOL, (e32, e64, ref_err)
    return e64 <= max(GRAD_TOL, 2 * ref_err), (e32, e64, ref_err)


def fwd_ok(img, ref32, faded: bool) -> bool:
    """Forward bar; cases with the support fade are ill-conditioned at the cutoff
    (exp(−q/2) − exp(−c²/2) cancels) and get 5e-5."""
    return rel_err(img, ref32) <= (5e-5 if faded else FWD_TOL)
