"""The reference extension's six native calls, served by this library.

The reference's CUDA wrapper (``cuda_render.py:52-174``) calls a JIT-built pybind module through
the module-level ``_EXT`` (``cuda_render._load_extension``, ``cuda_render.py:21-49``) with six
functions (``cuda/render_ext.cpp:303-317``):

* ``build_tile_index``       → ``ss_build_tile_index`` (count, scan, fill, sort; optional cull)
* ``forward_tiled``          → ``ss_forward_tiled`` on the caller's index
* ``backward_tiled``         → ``ss_backward_tiled`` on the caller's index
* ``forward``                → the untiled render: an index built here, then the tiled forward
* ``backward``               → the untiled backward: the index rebuilt, then the tiled backward
* ``backward_block_reduce``  → the same as ``backward`` (one backward serves both variants)

``Extension()`` is a drop-in for that module::

    from structsplat import cuda_render
    from structsplat_b200.reference_ext import Extension
    cuda_render._EXT = Extension()

after which ``render_cuda_exact`` and ``render_field(mode="cuda"/"cuda_tiled"/…)`` run on this
library through the reference's own autograd Function.

Argument checks and their messages follow ``render_ext.cpp:89-137`` (``RuntimeError`` like a
failed ``TORCH_CHECK``).  Tensors come back as the reference returns them: ``[out (H,W,3),
den (H,W)]`` and ``[grad_means, grad_conics, grad_colors, grad_opacities]`` (the last one
empty without opacities).  Every call runs on the current CUDA stream.  The fade tail is the
reference's ``expf(-0.5f·cutoff²)`` (``render_ext.cu:976``), evaluated by the C library.
The render kernels take tile sizes 16 and 32; an index of another tile size (the reference's
builder allows any ``tile_size² ≤ 1024``) is re-binned here at 32 before rendering, which gives
the same image (every pixel sums its Gaussians in ascending id either way).
"""
from __future__ import annotations

import torch

from . import _native
from .render import _stream

_RENDER_TILES = (16, 32)
_INTERNAL_TILE = 32


def _p(t):
    return t.data_ptr() if t is not None and t.numel() else None


def _check(cond: bool, message: str) -> None:
    if not cond:
        raise RuntimeError(message)


def _check_inputs(means, conics, colors, radii, opacities) -> None:
    """render_ext.cpp:94-125."""
    for name, t in (("means", means), ("conics", conics), ("colors", colors), ("radii", radii),
                    ("opacities", opacities)):
        _check(t.is_cuda, f"{name} must be a CUDA tensor")
        _check(t.is_contiguous(), f"{name} must be contiguous")
    for name, t in (("means", means), ("conics", conics), ("colors", colors)):
        _check(t.dtype == torch.float32, f"{name} must be float32")
    _check(radii.dtype == torch.int64, "radii must be int64")
    _check(opacities.numel() == 0 or opacities.dtype == torch.float32,
           "opacities must be empty or float32")
    _check(means.dim() == 2 and means.shape[1] == 2, "means must be (N, 2)")
    _check(conics.dim() == 2 and conics.shape[1] == 3, "conics must be (N, 3)")
    _check(colors.dim() == 2 and colors.shape[1] == 3, "colors must be (N, 3)")
    _check(radii.dim() == 2 and radii.shape[1] == 2, "radii must be (N, 2)")
    n = means.shape[0]
    _check(conics.shape[0] == n, "conics N must match means N")
    _check(colors.shape[0] == n, "colors N must match means N")
    _check(radii.shape[0] == n, "radii N must match means N")
    _check(opacities.numel() in (0, n), "opacities must be empty or length N")


def _check_tile_index(tile_gids, tile_offsets) -> None:
    """render_ext.cpp:127-137."""
    for name, t in (("tile_gids", tile_gids), ("tile_offsets", tile_offsets)):
        _check(t.is_cuda, f"{name} must be a CUDA tensor")
        _check(t.is_contiguous(), f"{name} must be contiguous")
        _check(t.dtype == torch.int32, f"{name} must be int32")
        _check(t.dim() == 1, f"{name} must be 1-D")


def _check_grad_inputs(grad_out, den, out) -> None:
    for name, t in (("grad_out", grad_out), ("den", den), ("out", out)):
        _check(t.is_cuda, f"{name} must be a CUDA tensor")
        _check(t.is_contiguous(), f"{name} must be contiguous")
        _check(t.dtype == torch.float32, f"{name} must be float32")
    _check(out.dim() == 3 and out.shape[2] == 3, "out must be (H, W, 3)")
    _check(grad_out.shape == out.shape, "grad_out must match out")
    _check(den.shape == out.shape[:2], "den must be (H, W)")


def _check_tile_size(tile_size: int) -> None:
    _check(tile_size > 0 and tile_size * tile_size <= 1024,
           "tile_size must be positive with tile_size^2 <= 1024")


class Extension:
    """The six functions of the reference's ``structsplat_render_ext`` module."""

    def __init__(self):
        _native.lib()  # raises when the CUDA library is missing: there is no fallback

    # -- helpers -----------------------------------------------------------------------------
    @staticmethod
    def _workspace(n: int, H: int, W: int, tile_size: int, capacity: int):
        size = _native.size_query("ss_reference_workspace_bytes", n, H, W, tile_size, capacity)
        return torch.empty(max(size, 256), dtype=torch.uint8, device="cuda"), size

    @staticmethod
    def _opacities(opacities):
        return opacities if opacities.numel() else None

    # -- the six calls ------------------------------------------------------------------------
    def build_tile_index(self, means, conics, radii, height, width, tile_size, ellipse_cull,
                         sigma_cutoff):
        """``[tile_gids int32, tile_offsets int32 (T+1)]`` (render_ext.cu:858-952).

        Two calls of ``ss_build_tile_index``: the first with capacity 0 leaves the entry total
        in ``offsets[T]`` (read back: the one host synchronisation the reference's build also
        makes, render_ext.cu:908-914), the second fills a list of exactly that size."""
        _check(means.is_cuda and conics.is_cuda and radii.is_cuda,
               "means, conics and radii must be CUDA tensors")
        _check(means.dtype == torch.float32 and conics.dtype == torch.float32,
               "means and conics must be float32")
        _check(radii.dtype == torch.int64, "radii must be int64")
        _check_tile_size(int(tile_size))
        H, W, ts = int(height), int(width), int(tile_size)
        means, conics, radii = means.contiguous(), conics.contiguous(), radii.contiguous()
        n = means.shape[0]
        tiles = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
        offsets = torch.zeros(tiles + 1, dtype=torch.int32, device=means.device)
        if n == 0 or tiles == 0:
            return [torch.empty(0, dtype=torch.int32, device=means.device), offsets]
        status = torch.zeros(1, dtype=torch.int32, device=means.device)
        ws, ws_bytes = self._workspace(n, H, W, ts, 0)
        args = (_p(means), _p(conics), _p(radii), n, H, W, ts, int(bool(ellipse_cull)),
                float(sigma_cutoff))
        _native.call("ss_build_tile_index", *args, None, 0, _p(offsets), _p(ws), ws_bytes,
                     _p(status), _stream())
        total = int(offsets[-1].item())
        gids = torch.empty(max(total, 1), dtype=torch.int32, device=means.device)
        if total:
            status.zero_()
            _native.call("ss_build_tile_index", *args, _p(gids), total, _p(offsets), _p(ws),
                         ws_bytes, _p(status), _stream())
        return [gids[:total], offsets]

    def forward_tiled(self, means, conics, colors, radii, opacities, tile_gids, tile_offsets,
                      height, width, normalize, eps, tile_size, support_fade, sigma_cutoff):
        """``[out (H,W,3), den (H,W)]`` rendered over the caller's index (render_ext.cu:1011-1063)."""
        _check_inputs(means, conics, colors, radii, opacities)
        _check_tile_index(tile_gids, tile_offsets)
        _check_tile_size(int(tile_size))
        H, W, ts = int(height), int(width), int(tile_size)
        if ts not in _RENDER_TILES:
            tile_gids, tile_offsets = self.build_tile_index(
                means, conics, radii, H, W, _INTERNAL_TILE, bool(support_fade), sigma_cutoff)
            ts = _INTERNAL_TILE
        tiles = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
        _check(tile_offsets.numel() == tiles + 1, "tile_offsets must have num_tiles + 1 entries")
        n = means.shape[0]
        out = torch.empty(H, W, 3, dtype=torch.float32, device=means.device)
        den = torch.empty(H, W, dtype=torch.float32, device=means.device)
        if H * W == 0:
            return [out, den]
        ws, ws_bytes = self._workspace(n, H, W, ts, tile_gids.numel())
        status = torch.zeros(1, dtype=torch.int32, device=means.device)
        _native.call("ss_forward_tiled", _p(means), _p(conics), _p(colors), _p(radii),
                     _p(self._opacities(opacities)), n, _p(tile_gids), tile_gids.numel(),
                     _p(tile_offsets), H, W, int(bool(normalize)), float(eps), ts,
                     int(bool(support_fade)), float(sigma_cutoff), _p(out), _p(den), _p(ws),
                     ws_bytes, _p(status), _stream())
        return [out, den]

    def backward_tiled(self, grad_out, means, conics, colors, radii, opacities, den, out,
                       tile_gids, tile_offsets, normalize, eps, tile_size, support_fade,
                       sigma_cutoff):
        """Gradients over the caller's index (render_ext.cu:1169-1231)."""
        _check_inputs(means, conics, colors, radii, opacities)
        _check_tile_index(tile_gids, tile_offsets)
        _check_grad_inputs(grad_out, den, out)
        _check_tile_size(int(tile_size))
        H, W = int(out.shape[0]), int(out.shape[1])
        ts = int(tile_size)
        if ts not in _RENDER_TILES:
            tile_gids, tile_offsets = self.build_tile_index(
                means, conics, radii, H, W, _INTERNAL_TILE, bool(support_fade), sigma_cutoff)
            ts = _INTERNAL_TILE
        n = means.shape[0]
        dev = means.device
        g_means = torch.zeros_like(means)
        g_conics = torch.zeros_like(conics)
        g_colors = torch.zeros_like(colors)
        has_op = opacities.numel() > 0
        g_opac = torch.zeros_like(opacities) if has_op else torch.empty(0, device=dev)
        if n == 0 or H * W == 0:
            return [g_means, g_conics, g_colors, g_opac]
        ws, ws_bytes = self._workspace(n, H, W, ts, tile_gids.numel())
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        _native.call("ss_backward_tiled", _p(grad_out), _p(means), _p(conics), _p(colors),
                     _p(radii), _p(self._opacities(opacities)), n, _p(den), _p(out),
                     _p(tile_gids), tile_gids.numel(), _p(tile_offsets), H, W,
                     int(bool(normalize)), float(eps), ts, int(bool(support_fade)),
                     float(sigma_cutoff), _p(g_means), _p(g_conics), _p(g_colors),
                     _p(g_opac) if has_op else None, _p(ws), ws_bytes, _p(status), _stream())
        return [g_means, g_conics, g_colors, g_opac]

    def forward(self, means, conics, colors, radii, opacities, height, width, normalize, eps,
                support_fade, sigma_cutoff):
        """The untiled render (render_ext.cu:956-1009): every Gaussian over its clipped
        rectangle.  Here the rectangles are binned into 32-px tiles first; the cull (exact
        under the full fade, the only fade this call has) drops only zero-weight pairs."""
        _check_inputs(means, conics, colors, radii, opacities)
        gids, offsets = self.build_tile_index(means, conics, radii, height, width,
                                              _INTERNAL_TILE, bool(support_fade), sigma_cutoff)
        return self.forward_tiled(means, conics, colors, radii, opacities, gids, offsets, height,
                                  width, normalize, eps, _INTERNAL_TILE, support_fade,
                                  sigma_cutoff)

    def backward(self, grad_out, means, conics, colors, radii, opacities, den, out, normalize,
                 eps, support_fade, sigma_cutoff):
        """The untiled backward (render_ext.cu:1067-1118).  The reference's wrapper keeps no
        index for the untiled path, so the index is rebuilt from the same inputs."""
        _check_inputs(means, conics, colors, radii, opacities)
        _check_grad_inputs(grad_out, den, out)
        gids, offsets = self.build_tile_index(means, conics, radii, out.shape[0], out.shape[1],
                                              _INTERNAL_TILE, bool(support_fade), sigma_cutoff)
        return self.backward_tiled(grad_out, means, conics, colors, radii, opacities, den, out,
                                   gids, offsets, normalize, eps, _INTERNAL_TILE, support_fade,
                                   sigma_cutoff)

    def backward_block_reduce(self, grad_out, means, conics, colors, radii, opacities, den, out,
                              normalize, eps, support_fade, sigma_cutoff):
        """The reference's block-reduced variant of the untiled backward (render_ext.cu:557-688)
        computes the same gradients; one backward serves both here."""
        return self.backward(grad_out, means, conics, colors, radii, opacities, den, out,
                             normalize, eps, support_fade, sigma_cutoff)
