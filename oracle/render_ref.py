"""CPU oracle of the clipped-support 2D Gaussian renderer (test infrastructure only).

Restates ``src/structsplat/render.py`` of the reference:

* ``support_rect``   ↔ ``_tile_bounds``        (render.py:62-78)
* ``visible_weight`` ↔ ``_support_weight``     (render.py:101-107)
* ``render``         ↔ ``_accumulate`` / ``render`` / ``render_additive`` (render.py:180-263)
* ``activity``       ↔ ``gaussian_activity``   (render.py:417-442)

Every (pixel, Gaussian) pair whose pixel lies in the Gaussian's clipped support rectangle is
evaluated exactly once; contributions are scattered with ``index_add`` so autograd yields the
reference's gradients.  Works in the dtype of ``means`` (float32 or float64).
"""
from __future__ import annotations

import math

import torch

DEFAULT_EPS = 1e-8
_PAIRS_PER_SLICE = 1 << 22


def support_rect(means: torch.Tensor, radii: torch.Tensor, H: int, W: int):
    """Support rectangle of each Gaussian clipped to the image (render.py:62-78).

    Centres are rounded half-to-even (``torch.round``).  Returns int64 tensors
    ``(x0, y0, tx, ty)``; a Gaussian with no in-image support has ``tx * ty == 0``.
    """
    cx = torch.round(means[:, 0].detach()).long()
    cy = torch.round(means[:, 1].detach()).long()
    rx = radii[:, 0].long()
    ry = radii[:, 1].long()
    x_lo = torch.clamp(cx - rx, min=0)
    x_hi = torch.clamp(cx + rx, max=W - 1)
    y_lo = torch.clamp(cy - ry, min=0)
    y_hi = torch.clamp(cy + ry, max=H - 1)
    tx = torch.clamp(x_hi - x_lo + 1, min=0)
    ty = torch.clamp(y_hi - y_lo + 1, min=0)
    tx = torch.where(ty > 0, tx, torch.zeros_like(tx))
    ty = torch.where(tx > 0, ty, torch.zeros_like(ty))
    return x_lo, y_lo, tx, ty


def pair_count(means, radii, H: int, W: int) -> int:
    """Number of in-rectangle (pixel, Gaussian) pairs: the renderer's algorithmic work."""
    _, _, tx, ty = support_rect(means, radii, H, W)
    return int((tx * ty).sum())


def fade_tail(sigma_cutoff: float, alpha: float) -> float:
    """Weight subtracted by the support fade: alpha·exp(−½ cutoff²) (render.py:101-107)."""
    return float(alpha) * math.exp(-0.5 * float(sigma_cutoff) ** 2)


def visible_weight(q: torch.Tensor, sigma_cutoff: float, alpha: float) -> torch.Tensor:
    """exp(−q/2), minus the fade tail and clamped at zero when the fade is on."""
    w = torch.exp(-0.5 * q)
    if alpha > 0.0:
        w = torch.clamp(w - fade_tail(sigma_cutoff, alpha), min=0.0)
    return w


def _slices(area: torch.Tensor, budget: int):
    """Consecutive Gaussian ranges whose summed support area stays within ``budget``."""
    n = area.shape[0]
    csum = torch.cumsum(area, 0)
    start, base = 0, 0
    while start < n:
        end = int(torch.searchsorted(csum, base + budget, right=True))
        end = min(max(end, start + 1), n)
        yield start, end
        base = int(csum[end - 1])
        start = end


def _expand(x0, y0, tx, area, s: int, e: int):
    """Flat pixel coordinates of the support rectangles of Gaussians [s, e)."""
    cnt = area[s:e]
    gid = torch.repeat_interleave(torch.arange(s, e), cnt)
    first = torch.cumsum(cnt, 0) - cnt
    k = torch.arange(int(cnt.sum())) - first[gid - s]
    width = tx[gid]
    return gid, x0[gid] + k % width, y0[gid] + k // width


def render(means, conics, colors, radii, H: int, W: int, opacities=None, normalize: bool = True,
           eps: float = DEFAULT_EPS, sigma_cutoff: float = 3.0, fade_alpha: float = 0.0,
           return_den: bool = False):
    """Reference image (H, W, 3): Σ w c / (Σ w + eps) (normalized) or Σ w c (additive).

    ``w = o · visible_weight(q)`` with ``q = a dx² + 2b dx dy + c dy²`` and ``d = pixel − mean``
    at integer pixel centres.  ``return_den`` also returns the raw weight sum (H, W) without eps
    — the denominator the reference CUDA extension hands to its backward.
    """
    if not (math.isfinite(eps) and eps > 0.0):
        raise ValueError(f"normalization_eps must be finite and > 0, got {eps}")
    dt = means.dtype
    num = torch.zeros(H * W, 3, dtype=dt)
    den = torch.zeros(H * W, dtype=dt)
    x0, y0, tx, ty = support_rect(means, radii, H, W)
    area = tx * ty
    for s, e in _slices(area, _PAIRS_PER_SLICE):
        gid, px, py = _expand(x0, y0, tx, area, s, e)
        if gid.numel() == 0:
            continue
        dx = px.to(dt) - means[gid, 0]
        dy = py.to(dt) - means[gid, 1]
        a, b, c = conics[gid, 0], conics[gid, 1], conics[gid, 2]
        q = a * dx * dx + 2.0 * b * dx * dy + c * dy * dy
        w = visible_weight(q, sigma_cutoff, fade_alpha)
        if opacities is not None:
            w = w * opacities[gid]
        pix = py * W + px
        num = num.index_add(0, pix, w[:, None] * colors[gid])
        den = den.index_add(0, pix, w)
    if normalize:
        img = (num / (den[:, None] + eps)).view(H, W, 3)
    else:
        img = num.view(H, W, 3)
    if return_den:
        return img, den.view(H, W)
    return img


def render_with_grads(means, conics, colors, radii, H: int, W: int, grad_out, opacities=None,
                      normalize: bool = True, eps: float = DEFAULT_EPS, sigma_cutoff: float = 3.0,
                      fade_alpha: float = 0.0):
    """Image, raw denominator and the gradients of ``Σ image · grad_out`` w.r.t. the inputs.

    Returns ``(image, den, {"means", "conics", "colors", "opacities"})`` where the opacity
    gradient is ``None`` without opacities.  This is the autograd of the reference equations,
    i.e. what ``_ExactRenderCuda.backward`` (cuda_render.py:123-174) must reproduce.
    """
    leaves = [t.detach().clone().requires_grad_(True) for t in (means, conics, colors)]
    op = None if opacities is None else opacities.detach().clone().requires_grad_(True)
    img, den = render(leaves[0], leaves[1], leaves[2], radii, H, W, opacities=op,
                      normalize=normalize, eps=eps, sigma_cutoff=sigma_cutoff,
                      fade_alpha=fade_alpha, return_den=True)
    inputs = leaves + ([op] if op is not None else [])
    grads = torch.autograd.grad(img, inputs, grad_out.to(img.dtype), allow_unused=True)
    names = ["means", "conics", "colors", "opacities"]
    out = {}
    for name, g, t in zip(names, list(grads) + [None] * (4 - len(grads)),
                          inputs + [None] * (4 - len(inputs))):
        if t is None:
            out[name] = None
        else:
            out[name] = torch.zeros_like(t) if g is None else g
    return img.detach(), den.detach(), out


@torch.no_grad()
def activity(means, conics, radii, H: int, W: int, sigma_cutoff: float = 3.0,
             fade_alpha: float = 0.0):
    """Per-Gaussian summed raw weight over its clipped support (render.py:417-442)."""
    dt = means.dtype
    act = torch.zeros(means.shape[0], dtype=dt)
    x0, y0, tx, ty = support_rect(means, radii, H, W)
    area = tx * ty
    for s, e in _slices(area, _PAIRS_PER_SLICE):
        gid, px, py = _expand(x0, y0, tx, area, s, e)
        if gid.numel() == 0:
            continue
        dx = px.to(dt) - means[gid, 0]
        dy = py.to(dt) - means[gid, 1]
        a, b, c = conics[gid, 0], conics[gid, 1], conics[gid, 2]
        q = a * dx * dx + 2.0 * b * dx * dy + c * dy * dy
        act.index_add_(0, gid, visible_weight(q, sigma_cutoff, fade_alpha))
    return act
