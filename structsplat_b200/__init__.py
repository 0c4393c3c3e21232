"""structsplat_b200 — StructSplat's tiled 2D Gaussian rasterizer, rebuilt for B200 (sm_100a).

Public entry points (all CUDA-only; the compute runs in ``_lib/libstructsplat_b200.so``):

* ``render_field`` / ``render_b200`` / ``build_tile_index`` — the reference's render call
  (``structsplat.render.render_field``, ``cuda_render.render_cuda_exact``) on the B200 kernels;
* ``render_gaussians`` — the fit path, straight from the RS field tensors;
* ``structure_tensor.compute`` — the placement operator J = G_ρ * (∇I∇Iᵀ);
* ``fit`` — graph-captured Adam fitting (single image and batched).
"""
from .render import build_tile_index, render_b200, render_field  # noqa: F401
from .field import render_gaussians  # noqa: F401

__all__ = ["build_tile_index", "render_b200", "render_field", "render_gaussians"]
__version__ = "0.1.0"
