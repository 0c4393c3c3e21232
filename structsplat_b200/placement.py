"""Density-weighted placement of a Gaussian field on the GPU.

Mirrors the reference's placement path for the ``density_random`` sampler:

* ``density_from_energy`` ↔ ``structsplat.density.density_from_energy`` (density.py:16-29)
* ``sample_candidates``   ↔ ``structsplat.density.sample_candidates``   (density.py:133-153)
* ``place_field``         ↔ ``structsplat.init.build_field`` with strategy ``aniso_onedge`` or
  ``iso_blue_noise`` and ``sampling_mode="density_random"`` (init.py:626-631, 778-847)

The sampler consumes explicit uniforms.  Given a numpy ``Generator`` (``rng=``) it draws them on
the host exactly as the reference's ``rng.choice`` + jitter do, so the points are the
reference's points; given a ``torch.Generator`` (``generator=``) it draws them on the device
(the same distribution, a different stream).  Everything else runs in the CUDA library.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native
from . import structure_tensor as st
from .render import _p, _stream

STRATEGIES = ("aniso_onedge", "iso_blue_noise")


def _workspace(H: int, W: int, device) -> tuple[torch.Tensor, int]:
    nbytes = _native.size_query("ss_placement_workspace_bytes", H, W)
    return torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device), nbytes


def energy_reference(energy: torch.Tensor) -> torch.Tensor:
    """structure_tensor.py:30-39 on the device: max(p99, 8·median) + 1e-12 (float64, 1 elem)."""
    e = torch.clamp_min(energy.detach().to(torch.float64).flatten(), 0.0)
    if e.numel() == 0:
        return torch.full((1,), 1e-12, dtype=torch.float64, device=energy.device)
    s, _ = torch.sort(e)
    n = s.numel()

    def lin(q):  # numpy's default (linear) percentile
        pos = (n - 1) * q
        lo = int(np.floor(pos))
        hi = min(lo + 1, n - 1)
        frac = pos - lo
        return s[lo] + (s[hi] - s[lo]) * frac
    med = (s[(n - 1) // 2] + s[n // 2]) / 2.0
    return (torch.maximum(lin(0.99), 8.0 * med) + 1e-12).reshape(1)


def density_from_energy(energy: torch.Tensor, base: float, power: float, ref=None):
    """Normalised density pmf (H, W) float64 from an energy map (H, W) float32 (CUDA)."""
    if not energy.is_cuda or energy.dtype != torch.float32 or energy.dim() != 2:
        raise ValueError("energy must be a 2-D CUDA float32 tensor")
    energy = energy.contiguous()
    H, W = energy.shape
    if ref is None:
        ref_t = energy_reference(energy)
    elif torch.is_tensor(ref):
        ref_t = ref.reshape(-1)[:1].to(device=energy.device, dtype=torch.float64)
    else:
        ref_t = torch.tensor([float(ref)], dtype=torch.float64, device=energy.device)
    out = torch.empty(H, W, dtype=torch.float64, device=energy.device)
    ws, nbytes = _workspace(H, W, energy.device)
    _native.call("ss_density_from_energy", _p(energy), H, W, float(base), float(power), _p(ref_t),
                 _p(out), _p(ws), nbytes, _stream())
    return out


def draw_uniforms(n: int, device, rng: np.random.Generator | None = None,
                  generator: torch.Generator | None = None) -> torch.Tensor:
    """The 3n uniforms of one sample_candidates call: n for the choice, then (n, 2) jitter."""
    if rng is not None:
        host = np.concatenate([rng.random(n), rng.random((n, 2)).ravel()])
        return torch.as_tensor(host, dtype=torch.float64).to(device)
    return torch.rand(3 * n, dtype=torch.float64, device=device, generator=generator)


def sample_candidates(density: torch.Tensor, n: int, rng: np.random.Generator | None = None,
                      generator: torch.Generator | None = None, uniforms=None,
                      return_index: bool = False):
    """``n`` sub-pixel positions (n, 2) float64 (x, y) distributed like ``density``."""
    if not density.is_cuda or density.dtype != torch.float64 or density.dim() != 2:
        raise ValueError("density must be a 2-D CUDA float64 tensor")
    density = density.contiguous()
    H, W = density.shape
    if uniforms is None:
        uniforms = draw_uniforms(n, density.device, rng=rng, generator=generator)
    if uniforms.numel() != 3 * n:
        raise ValueError(f"expected {3 * n} uniforms, got {uniforms.numel()}")
    pts = torch.empty(n, 2, dtype=torch.float64, device=density.device)
    idx = torch.empty(n, dtype=torch.int64, device=density.device) if return_index else None
    ws, nbytes = _workspace(H, W, density.device)
    _native.call("ss_sample_candidates", _p(density), H, W, _p(uniforms.contiguous()), int(n),
                 _p(pts), _p(idx), _p(ws), nbytes, _stream())
    return (pts, idx) if return_index else pts


def field_at_points(image, density, tensor: st.StructureTensor, pts, n_requested: int,
                    anisotropic: bool = True, max_axis_ratio: float = 6.0,
                    coherence_power: float = 1.0, init_scale_mult: float = 1.0) -> dict:
    """RS field tensors at the sampled points (build_field's post-sampling stage)."""
    H, W = density.shape
    n = pts.shape[0]
    dev = density.device
    f = {"means": torch.empty(n, 2, device=dev), "log_scales": torch.empty(n, 2, device=dev),
         "rotations": torch.empty(n, device=dev), "colors": torch.empty(n, 3, device=dev),
         "opacity_logits": None}
    img = image.contiguous()
    _native.call("ss_place_gaussians", _p(pts.contiguous()), n, _p(density),
                 _p(tensor.across_edge_angle.contiguous()), _p(tensor.coherence.contiguous()),
                 _p(img), H, W, int(anisotropic), float(max_axis_ratio), float(coherence_power),
                 float(init_scale_mult), int(n_requested), _p(f["means"]), _p(f["log_scales"]),
                 _p(f["rotations"]), _p(f["colors"]), _stream())
    return f


def place_field(image: torch.Tensor, n: int, strategy: str = "aniso_onedge", seed: int = 0,
                grad_sigma: float = 1.0, tensor_sigma: float = 2.0,
                density_base: float = 0.05, density_power: float = 1.0,
                max_axis_ratio: float = 6.0, coherence_power: float = 1.0,
                init_scale_mult: float = 1.0, numpy_rng: bool = True):
    """Structure tensor → density → seeded sampler → field, all on the GPU.

    With ``numpy_rng`` the sampler's uniforms come from ``np.random.default_rng(seed)`` exactly
    as the reference's ``build_field`` draws them (its first use of that generator), so the
    field is the reference's field; otherwise they come from a seeded ``torch.Generator``.
    Returns (field dict, StructureTensor, density).
    """
    if strategy not in STRATEGIES:
        raise ValueError(f"unsupported strategy {strategy!r}; expected one of {STRATEGIES}")
    if not image.is_cuda or image.dim() != 3 or image.shape[2] != 3:
        raise ValueError("image must be an (H, W, 3) CUDA tensor")
    image = image.to(torch.float32).contiguous()
    cfg = st.StructureTensorConfig(grad_sigma=grad_sigma, tensor_sigma=tensor_sigma)
    tensor = st.compute(image, cfg, sync_stats=False)
    density = density_from_energy(tensor.energy, density_base, density_power, ref=tensor.stats)
    if numpy_rng:
        pts = sample_candidates(density, n, rng=np.random.default_rng(seed))
    else:
        g = torch.Generator(device=image.device)
        g.manual_seed(seed)
        pts = sample_candidates(density, n, generator=g)
    field = field_at_points(image, density, tensor, pts, n,
                            anisotropic=strategy == "aniso_onedge", max_axis_ratio=max_axis_ratio,
                            coherence_power=coherence_power, init_scale_mult=init_scale_mult)
    return field, tensor, density
