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
