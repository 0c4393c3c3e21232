"""GPU structure tensor with the interface of ``structsplat.structure_tensor.compute``.

``compute(img, cfg)`` (structure_tensor.py:137-186) takes an (H,W,3) or (H,W) float image in
[0,1] and returns lam1, lam2, across-edge angle, coherence, energy, the flat/edge/corner label
map and the cached energy reference.  Here the image is a CUDA tensor (or an array, which is
uploaded) and the maps come back as CUDA tensors.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .render import _p, _stream

_OPERATORS = {"central": 0, "sobel": 1, "scharr": 2}
_COLOR_SPACES = {"luma": 0, "rgb": 1}


@dataclass
class StructureTensorConfig:
    """Same fields and defaults as the reference's ``StructureTensorConfig`` (config.py:70-78)."""
    grad_sigma: float = 1.0
    tensor_sigma: float = 2.0
    gradient_operator: str = "central"
    color_space: str = "luma"
    flat_frac: float = 0.02
    corner_frac: float = 0.15


@dataclass
class StructureTensor:
    lam1: torch.Tensor
    lam2: torch.Tensor
    across_edge_angle: torch.Tensor
    coherence: torch.Tensor
    energy: torch.Tensor
    label: torch.Tensor          # uint8: 0 flat, 1 edge, 2 corner
    energy_ref: float | None = None
    stats: torch.Tensor | None = None  # float64 [energy_ref, flat threshold, median, p99]

    @property
    def along_edge_angle(self) -> torch.Tensor:
        return self.across_edge_angle + np.pi / 2.0


def gaussian_taps(sigma: float) -> np.ndarray:
    """Normalised float32 Gaussian taps of radius max(1, round(3σ)) (structure_tensor.py:61-65),
    computed with the same float32 NumPy expression so the GPU blur uses identical weights."""
    radius = max(1, int(round(3.0 * sigma)))
    x = np.arange(-radius, radius + 1, dtype=np.float32)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return (k / k.sum()).astype(np.float32)


def compute(img, cfg: StructureTensorConfig | None = None, *, sync_stats: bool = True,
            device="cuda") -> StructureTensor:
    cfg = cfg or StructureTensorConfig()
    if cfg.gradient_operator not in _OPERATORS:
        raise ValueError(f"unknown gradient_operator {cfg.gradient_operator!r}; expected central, "
                         "sobel, or scharr")
    if cfg.color_space not in _COLOR_SPACES:
        raise ValueError(f"unknown color_space {cfg.color_space!r}; expected luma or rgb")
    if not torch.is_tensor(img):
        img = torch.as_tensor(np.asarray(img, dtype=np.float32), device=device)
    if not img.is_cuda:
        raise RuntimeError("the B200 structure tensor requires a CUDA tensor")
    img = img.to(torch.float32).contiguous()
    if img.dim() == 2:
        H, W, C = img.shape[0], img.shape[1], 1
    elif img.dim() == 3:
        H, W, C = img.shape
    else:
        raise ValueError("image must be (H, W) or (H, W, C)")
    dev = img.device
    tg = gaussian_taps(cfg.grad_sigma) if cfg.grad_sigma > 0 else np.zeros(1, np.float32)
    tt = gaussian_taps(cfg.tensor_sigma) if cfg.tensor_sigma > 0 else np.zeros(1, np.float32)
    rg = len(tg) // 2 if cfg.grad_sigma > 0 else 0
    rt = len(tt) // 2 if cfg.tensor_sigma > 0 else 0
    maps = torch.empty(5, H, W, device=dev, dtype=torch.float32)
    label = torch.empty(H, W, device=dev, dtype=torch.uint8)
    stats = torch.zeros(4, device=dev, dtype=torch.float64)
    ws_bytes = _native.size_query("ss_structure_tensor_workspace_bytes", H, W, C)
    ws = torch.empty(max(ws_bytes, 1), device=dev, dtype=torch.uint8)
    _native.call("ss_structure_tensor", _p(img), H, W, C,
                 tg.ctypes.data_as(ctypes.c_void_p), rg, tt.ctypes.data_as(ctypes.c_void_p), rt,
                 _OPERATORS[cfg.gradient_operator], _COLOR_SPACES[cfg.color_space],
                 float(cfg.flat_frac), float(cfg.corner_frac), _p(maps[0]), _p(maps[1]),
                 _p(maps[2]), _p(maps[3]), _p(maps[4]), _p(label), _p(stats), _p(ws), ws_bytes,
                 _stream())
    ref = float(stats[0].item()) if sync_stats else None
    return StructureTensor(maps[0], maps[1], maps[2], maps[3], maps[4], label, ref, stats)
