"""CPU oracle of the structure tensor J = G_ρ * (∇I ∇Iᵀ) (test infrastructure only).

Restates ``src/structsplat/structure_tensor.py`` (NumPy, float32 maps):

* ``luma``             ↔ ``to_luma``            (structure_tensor.py:54-58), Rec.709 weights
* ``gaussian_taps``    ↔ ``_gaussian_kernel``   (:61-65), radius max(1, round(3σ))
* ``blur``             ↔ ``gaussian_blur``      (:93-97), axis 0 then axis 1, reflect padding
* ``gradients``        ↔ ``gradients``          (:100-118), central / sobel / scharr
* ``energy_reference`` / ``flat_threshold``     (:30-51), float64 statistics
* ``compute``          ↔ ``compute``            (:137-186)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

LUMA = np.array([0.2126, 0.7152, 0.0722], dtype=np.float32)
ENERGY_REF_FLOOR_MULT = 8.0
FLAT_NOISE_MULT = 1.5


@dataclass
class TensorConfig:
    grad_sigma: float = 1.0
    tensor_sigma: float = 2.0
    gradient_operator: str = "central"
    color_space: str = "luma"
    flat_frac: float = 0.02
    corner_frac: float = 0.15


@dataclass
class TensorMaps:
    lam1: np.ndarray
    lam2: np.ndarray
    across_edge_angle: np.ndarray
    coherence: np.ndarray
    energy: np.ndarray
    label: np.ndarray
    energy_ref: float


def luma(img: np.ndarray) -> np.ndarray:
    img = np.asarray(img, dtype=np.float32)
    return img if img.ndim == 2 else img[..., :3] @ LUMA


def gaussian_taps(sigma: float) -> np.ndarray:
    r = max(1, int(round(3.0 * sigma)))
    x = np.arange(-r, r + 1, dtype=np.float32)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return (k / k.sum()).astype(np.float32)


def _conv_axis(a: np.ndarray, taps: np.ndarray, axis: int) -> np.ndarray:
    r = len(taps) // 2
    pad = [(r, r) if ax == axis else (0, 0) for ax in range(a.ndim)]
    padded = np.pad(a, pad, mode="reflect")
    acc = np.zeros_like(a)
    n = a.shape[axis]
    for i, w in enumerate(taps):
        window = [slice(None)] * a.ndim
        window[axis] = slice(i, i + n)
        acc += w * padded[tuple(window)]
    return acc


def blur(a: np.ndarray, sigma: float) -> np.ndarray:
    if sigma <= 0:
        return a
    taps = gaussian_taps(sigma)
    return _conv_axis(_conv_axis(a, taps, 0), taps, 1)


def _correlate3(a: np.ndarray, k: np.ndarray) -> np.ndarray:
    padded = np.pad(a, ((1, 1), (1, 1)), mode="reflect")
    acc = np.zeros_like(a, dtype=np.float32)
    h, w = a.shape
    for y in range(3):
        for x in range(3):
            acc += np.float32(k[y, x]) * padded[y:y + h, x:x + w]
    return acc


def gradients(g: np.ndarray, operator: str = "central"):
    """``(iy, ix)``; central differences are ``np.gradient`` (one-sided at the border)."""
    if operator == "central":
        iy, ix = np.gradient(g)
        return iy.astype(np.float32), ix.astype(np.float32)
    if operator == "sobel":
        kx = np.array([[-1, 0, 1], [-2, 0, 2], [-1, 0, 1]], dtype=np.float32) / 8.0
    elif operator == "scharr":
        kx = np.array([[-3, 0, 3], [-10, 0, 10], [-3, 0, 3]], dtype=np.float32) / 32.0
    else:
        raise ValueError(f"unknown gradient_operator {operator!r}")
    return _correlate3(g, kx.T), _correlate3(g, kx)


def energy_reference(energy: np.ndarray) -> float:
    e = np.maximum(np.asarray(energy, dtype=np.float64), 0.0)
    med = float(np.median(e)) if e.size else 0.0
    return float(max(np.percentile(e, 99.0), ENERGY_REF_FLOOR_MULT * med)) + 1e-12


def flat_threshold(energy: np.ndarray, flat_frac: float, ref: float) -> float:
    e = np.maximum(np.asarray(energy, dtype=np.float64), 0.0)
    med = float(np.median(e)) if e.size else 0.0
    return float(max(flat_frac * ref, FLAT_NOISE_MULT * med))


def compute(img: np.ndarray, cfg: TensorConfig | None = None) -> TensorMaps:
    cfg = cfg or TensorConfig()
    img = np.asarray(img, dtype=np.float32)
    if cfg.color_space == "rgb" and img.ndim == 3:
        chans = [blur(img[..., c], cfg.grad_sigma) for c in range(min(3, img.shape[-1]))]
    elif cfg.color_space in ("luma", "rgb"):
        chans = [blur(luma(img), cfg.grad_sigma)]
    else:
        raise ValueError(f"unknown color_space {cfg.color_space!r}")
    shape = chans[0].shape
    jxx = np.zeros(shape, np.float32)
    jxy = np.zeros(shape, np.float32)
    jyy = np.zeros(shape, np.float32)
    for ch in chans:
        iy, ix = gradients(ch, cfg.gradient_operator)
        jxx += ix * ix
        jxy += ix * iy
        jyy += iy * iy
    jxx = blur(jxx, cfg.tensor_sigma)
    jxy = blur(jxy, cfg.tensor_sigma)
    jyy = blur(jyy, cfg.tensor_sigma)
    half = 0.5 * (jxx + jyy)
    diff = 0.5 * (jxx - jyy)
    r = np.sqrt(diff * diff + jxy * jxy)
    lam1 = half + r
    lam2 = np.clip(half - r, 0.0, None)
    angle = 0.5 * np.arctan2(2.0 * jxy, jxx - jyy)
    energy = lam1 + lam2
    coherence = ((lam1 - lam2) / (energy + 1e-12)) ** 2
    ref = energy_reference(energy)
    label = np.zeros(shape, np.uint8)
    flat = energy < flat_threshold(energy, cfg.flat_frac, ref)
    corner = (lam2 > cfg.corner_frac * ref) & (~flat)
    label[~flat] = 1
    label[corner] = 2
    label[flat] = 0
    return TensorMaps(lam1.astype(np.float32), lam2.astype(np.float32),
                      angle.astype(np.float32), coherence.astype(np.float32),
                      energy.astype(np.float32), label, ref)
