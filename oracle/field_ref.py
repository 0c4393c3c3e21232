"""CPU oracle of the RS Gaussian-field parameterisation (test infrastructure only).

Restates ``src/structsplat/gaussians.py``:

* ``conics``         ↔ ``GaussianField.conics``         (gaussians.py:275-300)
* ``radii``          ↔ ``GaussianField.radii``          (gaussians.py:302-321)
* ``opacity_values`` ↔ ``GaussianField.opacity_values`` (gaussians.py:270-273)

A field is held as plain tensors: means (N,2), log_scales (N,2), rotations (N,),
colors (N,3) and optional opacity logits (N,).
"""
from __future__ import annotations

import torch


def conics(log_scales: torch.Tensor, rotations: torch.Tensor, dilation: float = 0.0):
    """Σ⁻¹ = R diag(1/(sx²+d), 1/(sy²+d)) Rᵀ as (N,3) ``[a, b, c]`` (differentiable)."""
    if dilation < 0.0:
        raise ValueError(f"dilation must be >= 0, got {dilation}")
    s = torch.exp(log_scales)
    inv_x = 1.0 / (s[:, 0] ** 2 + dilation)
    inv_y = 1.0 / (s[:, 1] ** 2 + dilation)
    cs = torch.cos(rotations)
    sn = torch.sin(rotations)
    a = cs * cs * inv_x + sn * sn * inv_y
    b = cs * sn * (inv_x - inv_y)
    c = sn * sn * inv_x + cs * cs * inv_y
    return torch.stack([a, b, c], dim=1)


@torch.no_grad()
def radii(log_scales: torch.Tensor, rotations: torch.Tensor, sigma_cutoff: float,
          dilation: float = 0.0):
    """int64 (N,2) half-widths ``ceil(cutoff·sqrt(Σ_xx)), ceil(cutoff·sqrt(Σ_yy))``, ≥ 1."""
    if dilation < 0.0:
        raise ValueError(f"dilation must be >= 0, got {dilation}")
    s2 = torch.exp(log_scales) ** 2 + dilation
    cs = torch.cos(rotations)
    sn = torch.sin(rotations)
    var_x = cs * cs * s2[:, 0] + sn * sn * s2[:, 1]
    var_y = sn * sn * s2[:, 0] + cs * cs * s2[:, 1]
    r = sigma_cutoff * torch.sqrt(torch.stack([var_x, var_y], dim=1))
    return torch.clamp(r.ceil().long(), min=1)


def opacity_values(logits):
    """sigmoid of the stored opacity logits, or ``None`` without opacities."""
    return None if logits is None else torch.sigmoid(logits)
