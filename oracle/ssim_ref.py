"""CPU oracle of the fit loss's SSIM term — test infrastructure, not product code.

Restates the reference's builtin SSIM (metrics.py:130-150): a normalised 11-tap Gaussian window
(sigma 1.5, metrics.py:65-84) applied as a horizontal then a vertical zero-padded pass per
channel, C1 = 0.01^2, C2 = 0.03^2, the mean of the SSIM map over channels and pixels; and the
fit loop's mix with the pixel loss, loss = (1 - w) pixel_loss + w (1 - SSIM) (fit.py:3244).
Differentiable with torch autograd, so the tests take its gradient as the reference's.  Pinned
by tests/golden/ssim_*.npz, made from the reference's own metrics.ssim.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F

C1, C2 = 0.01 ** 2, 0.03 ** 2


def window(win: int = 11, sigma: float = 1.5, device=None, dtype=torch.float32):
    """(horizontal, vertical) depthwise kernels for 3 channels of the normalised Gaussian."""
    x = torch.arange(win, device=device, dtype=dtype) - (win - 1) / 2.0
    g = torch.exp(-(x * x) / (2 * sigma * sigma))
    g = g / g.sum()
    return (g.reshape(1, 1, 1, win).repeat(3, 1, 1, 1), g.reshape(1, 1, win, 1).repeat(3, 1, 1, 1))


def _blur(x, wh, wv):
    pad = wh.shape[-1] // 2
    x = F.conv2d(x, wh, padding=(0, pad), groups=3)
    return F.conv2d(x, wv, padding=(pad, 0), groups=3)


def ssim(pred: torch.Tensor, target: torch.Tensor, win: int = 11, sigma: float = 1.5):
    """Mean SSIM of two (H, W, 3) images (0-dim tensor)."""
    p = pred.permute(2, 0, 1).unsqueeze(0)
    t = target.permute(2, 0, 1).unsqueeze(0)
    wh, wv = window(win, sigma, p.device, p.dtype)
    mu_p, mu_t = _blur(p, wh, wv), _blur(t, wh, wv)
    mu_p2, mu_t2, mu_pt = mu_p * mu_p, mu_t * mu_t, mu_p * mu_t
    sig_p = _blur(p * p, wh, wv) - mu_p2
    sig_t = _blur(t * t, wh, wv) - mu_t2
    sig_pt = _blur(p * t, wh, wv) - mu_pt
    num = (2 * mu_pt + C1) * (2 * sig_pt + C2)
    den = (mu_p2 + mu_t2 + C1) * (sig_p + sig_t + C2)
    return (num / den).mean()


def mixed_loss(pred, target, weight: float, pixel_loss: str = "l1"):
    """(1 - w) pixel_loss + w (1 - SSIM) with the fit loop's pixel losses (fit.py:800-814)."""
    d = pred - target
    if pixel_loss == "l1":
        pix = d.abs().mean(dim=2).mean()
    elif pixel_loss == "l2":
        pix = (d * d).mean(dim=2).mean()
    else:
        raise ValueError(f"unsupported pixel_loss {pixel_loss!r}")
    return (1 - weight) * pix + weight * (1 - ssim(pred, target))
