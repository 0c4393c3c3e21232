"""Graph-capturable rendering plans and the CUDA-graph-captured Adam fit.

``RenderPlan`` owns every buffer one forward + backward of an RS field needs (splat records,
tile offsets, a capacity-bounded tile list, workspaces, image, denominator, gradients), sized
once, so a step is a fixed sequence of library launches with no allocation and no host
synchronisation — exactly what a CUDA graph needs.  A step whose tile list would exceed the
capacity still renders exactly (truncated tiles scan every Gaussian) and raises
``SS_STATUS_INDEX_OVERFLOW`` in the plan's status word, which the host may read between replays
to re-plan with a larger capacity.

``fit`` runs the reference's plain fitting iteration (render → pixel MSE → backward → Adam,
``fit.py:3182-3351`` of the reference) through the batched fit path with one image, the whole
iteration captured in one CUDA graph.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import torch

from . import _native
from .render import (DEFAULT_EPS, RECORD_FLOATS, RENDER_TILE, _p, _stream, fade_tail, tile_grid,
                     validate_eps)

PARAM_NAMES = ("means", "log_scales", "rotations", "colors", "opacity_logits")


@dataclass
class RenderPlan:
    """Preallocated forward + backward of one RS field of ``n`` Gaussians on an H×W image."""
    n: int
    H: int
    W: int
    normalize: bool = True
    eps: float = DEFAULT_EPS
    sigma_cutoff: float = 3.0
    dilation: float = 0.0
    fade_alpha: float = 0.0
    has_opacity: bool = True
    capacity: int = 0
    deterministic: bool = False
    tile_size: int = RENDER_TILE
    device: torch.device = field(default_factory=lambda: torch.device("cuda"))
    # forward_backward in one tile pass (ss_render_forward_backward) instead of the forward and
    # backward tile kernels.  Off by default: at 1024x1024 with 100k Gaussians the fused pass
    # takes 0.103 ms against 0.051 + 0.057 ms alone, but the two kernels already overlap under
    # programmatic dependent launch, so the captured step is no faster (0.1365 vs 0.1345 ms).  A deterministic fused
    # plan leaves capacity-truncated tiles unrendered (SS_STATUS_DETERMINISTIC_TRUNCATED).
    fused: bool = False

    def __post_init__(self):
        if self.normalize:
            self.eps = validate_eps(self.eps)
        tiles_x, tiles_y = tile_grid(self.H, self.W, self.tile_size)
        self.T = tiles_x * tiles_y
        self.tail = fade_tail(self.sigma_cutoff, self.fade_alpha)
        self.cull = self.fade_alpha >= 1.0
        d, n = self.device, self.n
        f32 = dict(device=d, dtype=torch.float32)
        self.records = torch.empty(max(n, 1) * RECORD_FLOATS, **f32)
        self.offsets = torch.zeros(self.T + 1, device=d, dtype=torch.int32)
        self.idx_ws_bytes = _native.size_query("ss_tile_index_workspace_bytes", n, self.H, self.W,
                                               self.tile_size)
        self.idx_ws = torch.empty(max(self.idx_ws_bytes, 1), device=d, dtype=torch.uint8)
        if self.capacity <= 0:
            self.capacity = 1
        self.gids = torch.empty(self.capacity, device=d, dtype=torch.int32)
        self.bwd_ws_bytes = _native.size_query("ss_render_backward_workspace_bytes", n,
                                               self.capacity, self.H, self.W,
                                               int(self.deterministic))
        # the backward workspace and the status word share one allocation, which the step's
        # projection kernel clears (the moments in fast mode, the status word always)
        ws_len = (max(self.bwd_ws_bytes, 16) + 255) // 256 * 256
        self._step_block = torch.zeros(ws_len + 256, device=d, dtype=torch.uint8)
        self.bwd_ws = self._step_block[:ws_len]
        self._status_slot = self._step_block[ws_len:]
        self.status = self._status_slot[:4].view(torch.int32)
        self.image = torch.zeros(self.H, self.W, 3, **f32)
        self.den = torch.zeros(self.H, self.W, **f32)
        self.g_means = torch.zeros(n, 2, **f32)
        self.g_conics = torch.zeros(n, 3, **f32)
        self.g_colors = torch.zeros(n, 3, **f32)
        self.g_opac = torch.zeros(n, **f32)
        self.g_log_scales = torch.zeros(n, 2, **f32)
        self.g_rotations = torch.zeros(n, **f32)
        self.g_logits = torch.zeros(n, **f32)

    @classmethod
    def for_field(cls, params, H, W, headroom: float = 1.5, **kw):
        """Plan sized from the field's current tile-list total (one sync, at planning time)."""
        n = params["means"].shape[0]
        plan = cls(n=n, H=H, W=W, capacity=1, has_opacity=params.get("opacity_logits") is not None,
                   device=params["means"].device, **kw)
        plan.project(params)
        plan.count()
        total = int(plan.offsets[-1].item())
        return cls(n=n, H=H, W=W, capacity=int(total * headroom) + 4096,
                   has_opacity=plan.has_opacity, device=plan.device, **kw)

    # -- stages --------------------------------------------------------------------------
    def project(self, params):
        if self.n:
            _native.call("ss_project_rs", _p(params["means"]), _p(params["log_scales"]),
                         _p(params["rotations"]), _p(params["colors"]),
                         _p(params.get("opacity_logits") if self.has_opacity else None), self.n,
                         float(self.dilation), float(self.sigma_cutoff), self.H, self.W,
                         _p(self.records), None, None, _stream())

    def count(self):
        _native.call("ss_tile_index_count", _p(self.records), self.n, self.H, self.W,
                     self.tile_size, int(self.cull), float(self.sigma_cutoff), _p(self.offsets),
                     _p(self.idx_ws), self.idx_ws_bytes, _p(self.status), _stream())

    def project_count(self, params, clear_moments: bool = False):
        """project() and count() in one kernel (ss_project_rs_index_count), which also zeroes
        the status word and, with ``clear_moments`` in fast mode, the backward's moments."""
        region = self._step_block if clear_moments and not self.deterministic else self._status_slot
        _native.call("ss_project_rs_index_count", _p(params["means"]), _p(params["log_scales"]),
                     _p(params["rotations"]), _p(params["colors"]),
                     _p(params.get("opacity_logits") if self.has_opacity else None), self.n,
                     float(self.dilation), float(self.sigma_cutoff), self.H, self.W,
                     self.tile_size, int(self.cull), _p(self.records), _p(self.offsets),
                     _p(self.idx_ws), self.idx_ws_bytes, _p(region), region.numel(),
                     _p(self.status), _stream())

    def fill(self):
        _native.call("ss_tile_index_fill", _p(self.records), self.n, self.H, self.W,
                     self.tile_size, int(self.cull), float(self.sigma_cutoff), _p(self.offsets),
                     _p(self.gids), self.capacity, _p(self.idx_ws), self.idx_ws_bytes,
                     _p(self.status), _stream())

    def render(self):
        if self.H * self.W:
            _native.call("ss_render_forward", _p(self.records), self.n, _p(self.gids),
                         self.capacity, _p(self.offsets), self.H, self.W, self.tile_size,
                         int(self.normalize), float(self.eps), float(self.tail), _p(self.image),
                         _p(self.den), _p(self.status), _stream())

    def backward(self, grad_out, params, moments_zeroed: bool = False):
        """Gradients w.r.t. the RS parameters: the backward tile kernel into moments (fast) or
        entry partials (deterministic), then one per-Gaussian pass through the RS chain rule.
        ``moments_zeroed``: the caller already cleared the fast-mode moments."""
        if not self.n:
            return
        if not self.deterministic and not moments_zeroed:
            self.bwd_ws.zero_()
        self.backward_tiles(grad_out)
        self.finalize_rs(params)

    def render_input_grads(self, grad_out):
        """Gradients w.r.t. the render inputs (means, conics, colours, opacities) into
        g_means / g_conics / g_colors / g_opac, through the one-call ss_render_backward."""
        _native.call("ss_render_backward", _p(grad_out), _p(self.records), self.n, _p(self.den),
                     _p(self.image), _p(self.gids), self.capacity, _p(self.offsets), self.H,
                     self.W, self.tile_size, int(self.normalize), float(self.eps),
                     float(self.tail), int(self.has_opacity), _p(self.g_means),
                     _p(self.g_conics), _p(self.g_colors), _p(self.g_opac),
                     int(self.deterministic), _p(self.bwd_ws), self.bwd_ws_bytes,
                     _p(self.status), _stream())
        return self.g_means, self.g_conics, self.g_colors, self.g_opac

    def backward_tiles(self, grad_out):
        """Only the backward tile kernel (fast mode: adds into the moments), for timing."""
        _native.call("ss_render_backward_moments", _p(grad_out), None, _p(self.records), self.n,
                     _p(self.den), _p(self.image), _p(self.gids), self.capacity,
                     _p(self.offsets), self.H, self.W, self.tile_size, int(self.normalize),
                     float(self.eps), float(self.tail), int(self.deterministic), _p(self.bwd_ws),
                     self.bwd_ws_bytes, _p(self.status), _stream())

    def forward(self, params, clear_moments: bool = False):
        """Project, bin and render (the status word starts the step at zero; with
        ``clear_moments`` the fast-mode moments too, for a backward that follows)."""
        self.project_count(params, clear_moments)
        self.fill()
        self.render()
        return self.image

    def use_fused(self) -> bool:
        return bool(self.fused)

    def forward_backward(self, params, grad_out):
        """Image, den and the RS gradients for a grad_out known before the forward: project,
        bin, then one tile pass rendering and back-propagating each tile (or the forward and
        backward tile kernels one after the other), then the per-Gaussian RS pass."""
        # the projection kernel clears the moments, so the step's kernels follow one another
        # directly (each may start while its predecessor drains)
        if not self.use_fused():
            self.forward(params, clear_moments=True)
            self.backward(grad_out, params, moments_zeroed=True)
            return self.grads()
        self.project_count(params, clear_moments=True)
        self.fill()
        self.tile_pass(grad_out)
        if self.n:
            self.finalize_rs(params)
        return self.grads()

    def tile_pass(self, grad_out):
        """Only the fused forward + backward tile kernel (fast mode: adds into the moments)."""
        if self.H * self.W:
            _native.call("ss_render_forward_backward", _p(self.records), self.n, _p(self.gids),
                         self.capacity, _p(self.offsets), self.H, self.W, self.tile_size,
                         int(self.normalize), float(self.eps), float(self.tail), _p(grad_out),
                         _p(self.image), _p(self.den), int(self.deterministic), _p(self.bwd_ws),
                         self.bwd_ws_bytes, _p(self.status), _stream())

    def finalize_rs(self, params):
        _native.call("ss_render_backward_finalize_rs", _p(self.records), self.n, _p(self.gids),
                     self.capacity, _p(self.offsets), self.H, self.W, self.tile_size,
                     int(self.deterministic), _p(self.bwd_ws), _p(params["log_scales"]),
                     _p(params["rotations"]),
                     _p(params.get("opacity_logits") if self.has_opacity else None),
                     float(self.dilation), _p(self.g_means), _p(self.g_log_scales),
                     _p(self.g_rotations), _p(self.g_colors),
                     _p(self.g_logits if self.has_opacity else None), _stream())

    def grads(self):
        g = {"means": self.g_means, "log_scales": self.g_log_scales,
             "rotations": self.g_rotations, "colors": self.g_colors}
        if self.has_opacity:
            g["opacity_logits"] = self.g_logits
        return g

    def overflowed(self) -> bool:
        return bool(int(self.status.item()) & 1)


class CapturedStep:
    """A CUDA graph of ``fn()``; ``fn`` must only launch work on the current stream."""

    def __init__(self, fn, warmup: int = 2):
        self.fn = fn
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            for _ in range(warmup):
                fn()
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            fn()

    def replay(self):
        self.graph.replay()


def fit(params: dict, target: torch.Tensor, iters: int = 100, lr: float = 1e-2,
        normalize: bool = True, sigma_cutoff: float = 3.0, log_every: int = 0,
        graph: bool = True, settings=None, check_every: int = 50):
    """Adam fit of one RS field to ``target`` (H,W,3): the reference's plain fit iteration.

    ``params`` maps the five field names to CUDA float32 tensors (updated in place).  With no
    ``settings`` every parameter group uses learning rate ``lr`` and the loss is the pixel MSE.
    Returns a history dict: the PSNR of the pre-update render at every ``log_every`` iterations
    and ``final_psnr`` after the last update.  With ``graph=True`` one CUDA graph holds the
    whole iteration (index build, render + loss, backward, fused Adam update).
    """
    from .batch import FitSettings, fit_batch
    if settings is None:
        settings = FitSettings.uniform_lr(lr, normalize=normalize, sigma_cutoff=sigma_cutoff)
    h = fit_batch([params], [target], iters=iters, settings=settings, graph=graph,
                  log_every=log_every, check_every=check_every)
    out = {"iter": list(h["iter"]), "psnr": [p[0] for p in h["psnr"]],
           "final_psnr": h["final_psnr"][0], "replans": h["replans"],
           "overflowed": h["plan"].overflowed()}
    if not out["iter"] or out["iter"][-1] != iters:
        out["iter"].append(iters)
        out["psnr"].append(out["final_psnr"])
    return out
