"""CPU oracle of density-weighted placement (test infrastructure only).

Restates, in NumPy, the reference's placement path for the ``density_random`` sampler:

* ``density_from_energy`` ↔ ``density.density_from_energy``  (src/structsplat/density.py:16-29)
* ``sample_candidates``   ↔ ``density.sample_candidates``    (density.py:133-153) — written over
  explicit uniforms: numpy's ``Generator.choice(size, n, p=...)`` draws ``random(n)`` and
  searches them in the normalised cumulative sum, and the jitter is the next ``random((n, 2))``
  block; ``uniforms_for(seed, n)`` draws the same numbers;
* ``place_field``         ↔ ``init.build_field`` for strategies ``aniso_onedge`` /
  ``iso_blue_noise`` with ``sampling_mode="density_random"`` and the default scale, orientation,
  colour and opacity modes (init.py:39-82, 626-631, 778-847; gaussians.py:32-55).

Pinned against fixtures generated from the reference (tests/golden/make_golden.py, ``pl_*``).
"""
from __future__ import annotations

import math

import numpy as np
import torch


def energy_reference(energy: np.ndarray) -> float:
    """structure_tensor.py:24,30-39: max(p99, 8·median) + 1e-12 over max(e, 0) in float64."""
    e = np.maximum(np.asarray(energy, dtype=np.float64), 0.0)
    med = float(np.median(e)) if e.size else 0.0
    return float(max(np.percentile(e, 99.0), 8.0 * med)) + 1e-12


def density_from_energy(energy, base: float, power: float, ref: float | None = None):
    e = np.maximum(energy.astype(np.float64), 0.0)
    ref = energy_reference(e) if ref is None else float(ref)
    d = np.clip(e / ref, 0.0, 1.0) ** power
    d = base + (1.0 - base) * d
    s = d.sum()
    if not s > 0.0:
        return np.full(d.shape, 1.0 / d.size, dtype=np.float64)
    return (d / s).astype(np.float64)


def uniforms_for(seed: int, n: int) -> np.ndarray:
    """The 3n uniforms sample_candidates consumes from default_rng(seed): choice, then jitter."""
    rng = np.random.default_rng(seed)
    return np.concatenate([rng.random(n), rng.random((n, 2)).ravel()])


def _reflect(v, hi):
    v = np.abs(v)
    return hi - np.abs(hi - v)


def sample_candidates(density: np.ndarray, n: int, uniforms: np.ndarray):
    """Points (n,2) (x, y) float64 and the chosen pixel index, from explicit uniforms."""
    H, W = density.shape
    flat = density.ravel()
    flat = flat / flat.sum()
    cdf = flat.cumsum()
    cdf /= cdf[-1]
    idx = cdf.searchsorted(uniforms[:n], side="right")
    ys, xs = np.divmod(idx, W)
    jitter = uniforms[n:3 * n].reshape(n, 2) - 0.5
    xs = _reflect(xs + jitter[:, 0], W - 1.0)
    ys = _reflect(ys + jitter[:, 1], H - 1.0)
    return np.stack([xs, ys], axis=1).astype(np.float64), idx


def _nearest(map2d, pts):
    H, W = map2d.shape[:2]
    xi = np.clip(np.round(pts[:, 0]).astype(int), 0, W - 1)
    yi = np.clip(np.round(pts[:, 1]).astype(int), 0, H - 1)
    return map2d[yi, xi]


def _bilinear(img, pts):
    H, W = img.shape[:2]
    x = np.clip(pts[:, 0], 0, W - 1.001)
    y = np.clip(pts[:, 1], 0, H - 1.001)
    x0, y0 = np.floor(x).astype(int), np.floor(y).astype(int)
    x1, y1 = x0 + 1, y0 + 1
    fx, fy = (x - x0)[:, None], (y - y0)[:, None]
    c = (img[y0, x0] * (1 - fx) * (1 - fy) + img[y0, x1] * fx * (1 - fy)
         + img[y1, x0] * (1 - fx) * fy + img[y1, x1] * fx * fy)
    return c.astype(np.float32)


def place_field(img, density, across_edge_angle, coherence, pts, n_requested: int,
                anisotropic: bool = True, max_axis_ratio: float = 6.0,
                coherence_power: float = 1.0, init_scale_mult: float = 1.0):
    """The field build_field returns for the density_random sampler, as float32 arrays."""
    lam = np.maximum(n_requested * density, 1e-9)
    rmap = np.clip(np.sqrt(1.0 / (np.pi * lam)), 0.5, 20.0)
    spacing = _nearest(rmap, pts) * float(np.sqrt(np.pi))
    angles = _nearest(across_edge_angle + np.pi / 2.0, pts)
    if anisotropic:
        coh = np.clip(_nearest(coherence, pts), 0.0, 1.0) ** coherence_power
        ratios = 1.0 + (max_axis_ratio - 1.0) * coh
    else:
        ratios = np.ones(len(pts))
    ratios = np.maximum(ratios, 1.0)
    s_along = spacing * np.sqrt(ratios) * init_scale_mult
    s_across = spacing / np.sqrt(ratios) * init_scale_mult
    scales = np.clip(np.stack([s_along, s_across], 1), 1e-3, None)
    log_scales = torch.log(torch.as_tensor(scales, dtype=torch.float32)).numpy()
    return {"means": pts.astype(np.float32), "log_scales": log_scales,
            "rotations": np.asarray(angles, np.float32), "colors": _bilinear(img, pts)}


def spacing_per_radius() -> float:
    return math.sqrt(math.pi)
