"""Seeded synthetic targets and Gaussian fields for the benchmark workloads.

No public dataset is involved.  The target generator draws sinusoid gratings of random
orientation, random filled polygons and Gaussian noise; the field generator draws the
distribution the benchmark workloads are quoted on (means uniform over the image,
σ = exp(N(ln 2, 0.5)), θ ~ U[0, π), RGB ~ U[0,1]³, opacity = sigmoid(N(0, 1)), stored as logits
the way ``GaussianField`` stores them, ``src/structsplat/gaussians.py:15-29,270-273``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _fill_polygon(img: np.ndarray, verts: np.ndarray, colour: np.ndarray) -> None:
    """Paint a polygon (even-odd rule at pixel centres) over ``img`` in place."""
    H, W, _ = img.shape
    x_lo = max(int(np.floor(verts[:, 0].min())), 0)
    x_hi = min(int(np.ceil(verts[:, 0].max())), W - 1)
    y_lo = max(int(np.floor(verts[:, 1].min())), 0)
    y_hi = min(int(np.ceil(verts[:, 1].max())), H - 1)
    if x_lo > x_hi or y_lo > y_hi:
        return
    ys, xs = np.mgrid[y_lo:y_hi + 1, x_lo:x_hi + 1].astype(np.float64)
    inside = np.zeros(xs.shape, dtype=bool)
    n = len(verts)
    for k in range(n):
        xa, ya = verts[k]
        xb, yb = verts[(k + 1) % n]
        crosses = (ya > ys) != (yb > ys)
        with np.errstate(divide="ignore", invalid="ignore"):
            x_at = xa + (ys - ya) * (xb - xa) / (yb - ya)
        inside ^= crosses & (xs < x_at)
    img[y_lo:y_hi + 1, x_lo:x_hi + 1][inside] = colour


def make_target(H: int, W: int, seed: int, n_gratings: int = 8, n_polygons: int = 20,
                noise_std: float = 0.02) -> np.ndarray:
    """H×W×3 float32 image in [0, 1]: gratings (period 8–64 px) + polygons + N(0, σ²) noise."""
    rng = np.random.default_rng(seed)
    ys, xs = np.mgrid[0:H, 0:W].astype(np.float32)
    img = np.full((H, W, 3), 0.5, np.float32)
    for _ in range(n_gratings):
        theta = rng.uniform(0.0, math.pi)
        period = rng.uniform(8.0, 64.0)
        phase = rng.uniform(0.0, 2 * math.pi)
        weight = rng.uniform(-1.0, 1.0, 3).astype(np.float32) * (0.35 / n_gratings ** 0.5)
        wave = np.sin((xs * math.cos(theta) + ys * math.sin(theta)) * (2 * math.pi / period)
                      + phase).astype(np.float32)
        img += wave[..., None] * weight
    span = 0.5 * min(H, W)
    for _ in range(n_polygons):
        centre = rng.uniform([0.0, 0.0], [W, H])
        k = int(rng.integers(3, 9))
        ang = np.sort(rng.uniform(0.0, 2 * math.pi, k))
        rad = rng.uniform(0.05, 0.35, k) * span
        verts = np.stack([centre[0] + rad * np.cos(ang), centre[1] + rad * np.sin(ang)], 1)
        _fill_polygon(img, verts, rng.uniform(0.0, 1.0, 3).astype(np.float32))
    img += rng.normal(0.0, noise_std, img.shape).astype(np.float32)
    return np.clip(img, 0.0, 1.0).astype(np.float32)


@dataclass
class FieldArrays:
    """Gaussian field in the reference's tensor layout (numpy, float32)."""
    means: np.ndarray           # (N, 2) pixel coordinates
    log_scales: np.ndarray      # (N, 2)
    rotations: np.ndarray       # (N,)
    colors: np.ndarray          # (N, 3)
    opacity_logits: np.ndarray  # (N,)

    @property
    def n(self) -> int:
        return int(self.means.shape[0])


def make_field(H: int, W: int, n: int, seed: int, log_sigma_mean: float = math.log(2.0),
               log_sigma_std: float = 0.5) -> FieldArrays:
    """Field with uniform means, log-normal σ, uniform angle/colour and logistic opacity."""
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(0.0, W, n), rng.uniform(0.0, H, n)], 1).astype(np.float32)
    log_scales = rng.normal(log_sigma_mean, log_sigma_std, (n, 2)).astype(np.float32)
    rotations = rng.uniform(0.0, math.pi, n).astype(np.float32)
    colors = rng.uniform(0.0, 1.0, (n, 3)).astype(np.float32)
    logits = rng.normal(0.0, 1.0, n).astype(np.float32)
    return FieldArrays(means, log_scales, rotations, colors, logits)


def make_stress_field(H: int, W: int, n: int, seed: int, along_edge_angle: np.ndarray,
                      log_sigma_std: float = 1.2, elongated_frac: float = 0.3,
                      aspect_range=(5.0, 50.0)) -> FieldArrays:
    """Heavy-tailed stress field: σ = exp(N(ln 2, 1.2)) per Gaussian, and a fraction of
    elongated Gaussians (aspect ratio U[5, 50], same area) aligned with ``along_edge_angle``
    (H, W) read at the pixel nearest their mean; the rest as ``make_field``.  The heavy tail
    gives tile lists from a few entries to ~10⁴."""
    f = make_field(H, W, n, seed, log_sigma_std=log_sigma_std)
    rng = np.random.default_rng(seed + 7919)
    sigma = rng.normal(math.log(2.0), log_sigma_std, n).astype(np.float32)
    f.log_scales[:, 0] = sigma
    f.log_scales[:, 1] = sigma
    elong = rng.random(n) < elongated_frac
    k = int(elong.sum())
    half_log_ar = 0.5 * np.log(rng.uniform(aspect_range[0], aspect_range[1], k)).astype(np.float32)
    f.log_scales[elong, 0] += half_log_ar
    f.log_scales[elong, 1] -= half_log_ar
    xi = np.clip(np.round(f.means[elong, 0]).astype(int), 0, W - 1)
    yi = np.clip(np.round(f.means[elong, 1]).astype(int), 0, H - 1)
    f.rotations[elong] = np.asarray(along_edge_angle, np.float32)[yi, xi]
    return f
