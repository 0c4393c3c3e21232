"""Host side of the B200 renderer: the reference's render call, re-pointed at the CUDA library.

Mirrors the reference interface so it drops in behind the fitting loop:

* ``render_field``      ↔ ``structsplat.render.render_field``      (render.py:319-414)
* ``render_b200``       ↔ ``structsplat.cuda_render.render_cuda_exact`` (cuda_render.py:256-294)
* ``build_tile_index``  ↔ the extension's ``build_tile_index``     (render_ext.cu:858-952)
* ``_B200Render``       ↔ ``_ExactRenderCuda``                     (cuda_render.py:52-174)

Tensor contract (render_ext.cpp:89-137): means (N,2) f32, conics (N,3) f32 ``[a, b, c]`` with
``q = a dx² + 2b dx dy + c dy²``, colors (N,3) f32, radii (N,2) int64, opacities (N,) f32 or
None; CUDA tensors only — there is no CPU fallback.  Everything runs on the current CUDA stream.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from . import _native

DEFAULT_EPS = 1e-8
RECORD_FLOATS = 16  # one 64-byte splat record

NORMALIZED_MODES = ("b200", "b200_normalized", "normalized", "cuda", "cuda_normalized",
                    "cuda_block_reduce", "cuda_tiled", "cuda_tiled_normalized")
ADDITIVE_MODES = ("b200_additive", "additive", "cuda_additive", "cuda_tiled_additive")


def _p(t):
    """Device address of a tensor as a plain int (ctypes passes it as ``void*``), None → NULL."""
    return None if t is None else t.data_ptr()


_RAW_STREAM = getattr(torch._C, "_cuda_getCurrentRawStream", None)
_DEVICE = getattr(torch._C, "_cuda_getDevice", None)


def _stream():
    """The current CUDA stream of the current device as a raw ``cudaStream_t`` address.

    Read through torch's C getters where this torch has them: ``torch.cuda.current_stream()``
    builds a Python Stream object and re-resolves the device on every call, which costs several
    microseconds per library call on the eager path."""
    if _RAW_STREAM is None or _DEVICE is None:
        return torch.cuda.current_stream().cuda_stream
    if not torch.cuda.is_initialized():
        torch.cuda.init()
    return _RAW_STREAM(_DEVICE())


def validate_eps(value: float) -> float:
    """Same rule as render.py:33-37."""
    eps = float(value)
    if not math.isfinite(eps) or eps <= 0.0:
        raise ValueError(f"normalization_eps must be finite and > 0, got {value}")
    return eps


def resolve_fade_alpha(support_fade: bool, support_fade_alpha=None) -> float:
    """render.py:94-98: None → 1 with the fade on, 0 off; otherwise clamped to [0, 1]."""
    if support_fade_alpha is None:
        return 1.0 if support_fade else 0.0
    return max(0.0, min(1.0, float(support_fade_alpha)))


def fade_tail(sigma_cutoff: float, alpha: float) -> float:
    """alpha·exp(−½ cutoff²) as the float32 the reference subtracts (render.py:101-107)."""
    if alpha <= 0.0:
        return 0.0
    return float(np.float32(alpha * math.exp(-0.5 * float(sigma_cutoff) ** 2)))


def tile_grid(H: int, W: int, tile_size: int) -> tuple[int, int]:
    if tile_size <= 0 or tile_size * tile_size > 1024:
        raise ValueError("tile_size must be positive with tile_size^2 <= 1024")
    return (W + tile_size - 1) // tile_size, (H + tile_size - 1) // tile_size


def _check_cuda_f32(means, conics, colors):
    if not means.is_cuda:
        raise RuntimeError("StructSplat B200 renderer requires CUDA tensors; pass device='cuda'.")
    if means.dtype != torch.float32 or conics.dtype != torch.float32 or \
            colors.dtype != torch.float32:
        raise RuntimeError("StructSplat B200 renderer supports float32 tensors only.")


def _check_shapes(means, conics, colors, radii, opacities):
    n = means.shape[0]
    if means.dim() != 2 or means.shape[1] != 2:
        raise ValueError("means must be (N, 2)")
    if conics.shape != (n, 3):
        raise ValueError("conics must be (N, 3)")
    if colors.shape != (n, 3):
        raise ValueError("colors must be (N, 3)")
    if radii.shape != (n, 2) or radii.dtype != torch.int64:
        raise ValueError("radii must be (N, 2) int64")
    if opacities is not None and opacities.numel() not in (0, n):
        raise ValueError("opacities must be empty or length N")
    for t in (conics, colors, radii):
        if t.device != means.device:
            raise ValueError("all inputs must be on the same device")


@dataclass
class TileIndex:
    """Per-tile Gaussian lists: tile t is ``gids[offsets[t]:offsets[t+1]]`` (ascending ids)."""
    gids: torch.Tensor      # int32 [entries]
    offsets: torch.Tensor   # int32 [T+1]
    tile_size: int
    status: torch.Tensor    # int32 [1] device status word

    @property
    def capacity(self) -> int:
        return int(self.gids.numel())


def pack_records(means, conics, colors, radii, opacities, H: int, W: int) -> torch.Tensor:
    n = means.shape[0]
    rec = torch.empty(max(n, 1) * RECORD_FLOATS, device=means.device, dtype=torch.float32)
    if n:
        _native.call("ss_pack_splats", _p(means), _p(conics), _p(colors), _p(radii),
                     _p(opacities), n, H, W, _p(rec), _stream())
    return rec


class _CapacityCache:
    """Per-problem capacity for the tile index, so steady-state calls never wait on the host.

    The first call for a (device, N, H, W, tile size, cull) key reads the entry total back
    (one sync, as the reference's build does at render_ext.cu:908-914) and keeps 25 % headroom.
    Later calls reuse that capacity and copy their own total to pinned memory asynchronously;
    the next call reads it (only once its copy has completed) and grows the capacity if
    needed.  A call whose total exceeds the capacity still renders exactly: the kernels scan
    every Gaussian for the truncated tiles.
    """

    def __init__(self):
        self.entries = {}

    def capacity(self, key, offsets) -> int:
        ent = self.entries.get(key)
        if ent is None:
            total = int(offsets[-1].item())
            cap = int(total * 1.25) + 1024
            host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
            ent = self.entries[key] = {"cap": cap, "host": host, "event": None,
                                       "recorder": torch.cuda.Event()}
        elif ent["event"] is not None and ent["event"].query():
            seen = int(ent["host"][0])
            if seen > ent["cap"]:
                ent["cap"] = int(seen * 1.25) + 1024
        ent["host"].copy_(offsets[-1:], non_blocking=True)
        ent["recorder"].record()
        ent["event"] = ent["recorder"]
        return ent["cap"]


CAPACITY = _CapacityCache()


class EagerPlan:
    """Buffers of one problem (device, N, H, W, tile size, cull) for the eager autograd path,
    kept between calls: splat records, tile offsets and list, index workspace, and the fast
    backward's moments and status word in one block that the step clears.  A fit loop renders
    the same problem every iteration, so a forward + backward then allocates only its outputs
    and makes five library calls.

    The plan holds the state of the last forward that used it (``generation``).  A backward
    whose forward has been followed by another forward on the same plan (two renders before one
    backward) rebuilds its records and index from its saved inputs instead.  The list capacity
    starts at the first call's entry total (one host read) with headroom; each call copies its
    status word to pinned memory, and a later call that finds an overflow there re-reads the
    total and grows the list (the overflowing call itself was exact: its truncated tiles scan
    every Gaussian)."""

    HEADROOM = 1.5

    def __init__(self, n: int, H: int, W: int, tile_size: int, cull: bool, sigma_cutoff: float,
                 device):
        self.n, self.H, self.W, self.ts = n, H, W, tile_size
        self.cull, self.cutoff = bool(cull), float(sigma_cutoff)
        tiles_x, tiles_y = tile_grid(H, W, tile_size)
        self.T = tiles_x * tiles_y
        d = device
        self.records = torch.empty(max(n, 1) * RECORD_FLOATS, device=d, dtype=torch.float32)
        self.offsets = torch.zeros(self.T + 1, device=d, dtype=torch.int32)
        self.idx_ws_bytes = _native.size_query("ss_tile_index_workspace_bytes", n, H, W,
                                               tile_size)
        self.idx_ws = torch.empty(max(self.idx_ws_bytes, 1), device=d, dtype=torch.uint8)
        self.capacity = 0
        self.gids = None
        self.generation = 0
        self.moments_used = False
        self.host_status = torch.zeros(1, dtype=torch.int32, pin_memory=True)
        self.status_event = torch.cuda.Event()  # re-recorded by every call
        self.event = None
        self._size_list(1)

    def _size_list(self, capacity: int):
        self.capacity = int(capacity)
        d = self.records.device
        self.gids = torch.empty(max(self.capacity, 1), device=d, dtype=torch.int32)
        self.bwd_ws_bytes = _native.size_query("ss_render_backward_workspace_bytes", self.n,
                                               self.capacity, self.H, self.W, 0)
        ws_len = (max(self.bwd_ws_bytes, 16) + 255) // 256 * 256
        self.step_block = torch.zeros(ws_len + 256, device=d, dtype=torch.uint8)
        self.bwd_ws = self.step_block[:ws_len]
        self.status = self.step_block[ws_len:ws_len + 4].view(torch.int32)

    def ensure_capacity(self):
        """After the count: size the list on first use, or grow it after an overflow seen in
        an earlier call's status (both read the entry total back)."""
        grow = self.gids is None or self.capacity <= 1
        if not grow and self.event is not None and self.event.query():
            grow = bool(int(self.host_status[0]) & 1)
            self.event = None
        if grow:
            total = int(self.offsets[-1].item())
            if total > self.capacity or self.capacity <= 1:
                self._size_list(int(total * self.HEADROOM) + 4096)
                self.step_block.zero_()

    def note_status(self):
        self.host_status.copy_(self.status, non_blocking=True)
        self.status_event.record()
        self.event = self.status_event


class _EagerPlans:
    """One EagerPlan per problem key; a handful of keys at most in a fit."""

    def __init__(self, limit: int = 8):
        self.plans = {}
        self.limit = limit

    def get(self, n, H, W, tile_size, cull, sigma_cutoff, device) -> EagerPlan:
        key = (device.index, n, H, W, tile_size, bool(cull), float(sigma_cutoff))
        plan = self.plans.get(key)
        if plan is None:
            if len(self.plans) >= self.limit:
                self.plans.pop(next(iter(self.plans)))
            plan = self.plans[key] = EagerPlan(n, H, W, tile_size, cull, sigma_cutoff, device)
        return plan


EAGER_PLANS = _EagerPlans()


def index_from_records(records, n: int, H: int, W: int, tile_size: int = 16,
                       ellipse_cull: bool = False, sigma_cutoff: float = 3.0,
                       capacity: int | None = None, exact: bool = False) -> TileIndex:
    """Count → scan → fill → sort.  ``exact`` reads the entry total back (one device→host sync)
    and sizes the list exactly; otherwise the capacity comes from ``capacity`` or the
    per-problem cache."""
    tiles_x, tiles_y = tile_grid(H, W, tile_size)
    T = tiles_x * tiles_y
    dev = records.device
    offsets = torch.empty(T + 1, device=dev, dtype=torch.int32)
    status = torch.zeros(1, device=dev, dtype=torch.int32)
    ws_bytes = _native.size_query("ss_tile_index_workspace_bytes", n, H, W, tile_size)
    ws = torch.empty(max(ws_bytes, 1), device=dev, dtype=torch.uint8)
    _native.call("ss_tile_index_count", _p(records), n, H, W, tile_size, int(ellipse_cull),
                 float(sigma_cutoff), _p(offsets), _p(ws), ws_bytes, _p(status), _stream())
    if T == 0:
        capacity = 0
    elif exact:
        capacity = int(offsets[-1].item())
    elif capacity is None:
        key = (dev.index, n, H, W, tile_size, bool(ellipse_cull))
        capacity = CAPACITY.capacity(key, offsets)
    gids = torch.empty(max(capacity, 1), device=dev, dtype=torch.int32)
    _native.call("ss_tile_index_fill", _p(records), n, H, W, tile_size, int(ellipse_cull),
                 float(sigma_cutoff), _p(offsets), _p(gids), int(capacity), _p(ws), ws_bytes,
                 _p(status), _stream())
    return TileIndex(gids[:capacity], offsets, tile_size, status)


def build_tile_index(means, conics, radii, H: int, W: int, tile_size: int = 16,
                     ellipse_cull: bool = False, sigma_cutoff: float = 3.0):
    """``(gids int32 [entries], offsets int32 [T+1])`` like the extension's build_tile_index."""
    if not means.is_cuda:
        raise RuntimeError("StructSplat B200 renderer requires CUDA tensors; pass device='cuda'.")
    tile_grid(H, W, tile_size)
    means = means.detach().contiguous()
    conics = conics.detach().contiguous().to(torch.float32)
    radii = radii.contiguous()
    rec = pack_records(means.to(torch.float32), conics, conics, radii, None, H, W)
    idx = index_from_records(rec, means.shape[0], H, W, tile_size, ellipse_cull, sigma_cutoff,
                             exact=True)
    return idx.gids, idx.offsets


def _forward(records, n, index: TileIndex, H, W, normalize, eps, tail, dev):
    out = torch.empty(H, W, 3, device=dev, dtype=torch.float32)
    den = torch.empty(H, W, device=dev, dtype=torch.float32)
    if H * W:
        _native.call("ss_render_forward", _p(records), n, _p(index.gids), index.capacity,
                     _p(index.offsets), H, W, index.tile_size, int(normalize), float(eps),
                     float(tail), _p(out), _p(den), _p(index.status), _stream())
    return out, den


def _backward(grad_out, records, n, den, out, index: TileIndex, H, W, normalize, eps, tail,
              has_opacity, deterministic, dev):
    g_means = torch.empty(n, 2, device=dev, dtype=torch.float32)
    g_conics = torch.empty(n, 3, device=dev, dtype=torch.float32)
    g_colors = torch.empty(n, 3, device=dev, dtype=torch.float32)
    g_opac = torch.empty(n, device=dev, dtype=torch.float32) if has_opacity else None
    ws_bytes = _native.size_query("ss_render_backward_workspace_bytes", n, index.capacity, H, W,
                                  int(deterministic))
    ws = torch.empty(max(ws_bytes, 16), device=dev, dtype=torch.uint8)
    _native.call("ss_render_backward", _p(grad_out), _p(records), n, _p(den), _p(out),
                 _p(index.gids), index.capacity, _p(index.offsets), H, W, index.tile_size,
                 int(normalize), float(eps), float(tail), int(has_opacity), _p(g_means),
                 _p(g_conics), _p(g_colors), _p(g_opac), int(deterministic), _p(ws), ws_bytes,
                 _p(index.status), _stream())
    return g_means, g_conics, g_colors, g_opac


class _B200Render(Function):
    """Autograd Function with the slots of ``_ExactRenderCuda`` (cuda_render.py:52-174)."""

    @staticmethod
    def forward(ctx, means, conics, colors, radii, opacities, H, W, normalize, eps, tile_size,
                tail, cull, sigma_cutoff, deterministic):
        n = means.shape[0]
        means, conics, colors = means.contiguous(), conics.contiguous(), colors.contiguous()
        radii = radii.contiguous()
        has_op = opacities is not None and opacities.numel() > 0
        op = opacities.contiguous() if has_op else None
        ctx.meta = (n, H, W, bool(normalize), float(eps), int(tile_size), float(tail), has_op,
                    bool(deterministic), bool(cull), float(sigma_cutoff))
        if not deterministic and n and H * W:
            # the fast path: the problem's buffers persist between calls (EagerPlan)
            plan = EAGER_PLANS.get(n, H, W, tile_size, cull, sigma_cutoff, means.device)
            plan.step_block.zero_()  # fast moments and the status word
            stream = _stream()
            _native.call("ss_pack_splats", _p(means), _p(conics), _p(colors), _p(radii), _p(op),
                         n, H, W, _p(plan.records), stream)
            _native.call("ss_tile_index_count", _p(plan.records), n, H, W, tile_size, int(cull),
                         float(sigma_cutoff), _p(plan.offsets), _p(plan.idx_ws),
                         plan.idx_ws_bytes, _p(plan.status), stream)
            plan.ensure_capacity()
            _native.call("ss_tile_index_fill", _p(plan.records), n, H, W, tile_size, int(cull),
                         float(sigma_cutoff), _p(plan.offsets), _p(plan.gids), plan.capacity,
                         _p(plan.idx_ws), plan.idx_ws_bytes, _p(plan.status), stream)
            out = torch.empty(H, W, 3, device=means.device, dtype=torch.float32)
            den = torch.empty(H, W, device=means.device, dtype=torch.float32)
            _native.call("ss_render_forward", _p(plan.records), n, _p(plan.gids), plan.capacity,
                         _p(plan.offsets), H, W, tile_size, int(normalize), float(eps),
                         float(tail), _p(out), _p(den), _p(plan.status), stream)
            plan.note_status()
            plan.generation += 1
            plan.moments_used = False
            ctx.plan, ctx.generation = plan, plan.generation
            ctx.save_for_backward(out, den, means, conics, colors, radii, op)
            return out
        rec = pack_records(means, conics, colors, radii, op, H, W)
        index = index_from_records(rec, n, H, W, tile_size, cull, sigma_cutoff,
                                   exact=bool(deterministic))
        out, den = _forward(rec, n, index, H, W, normalize, eps, tail, means.device)
        ctx.plan = None
        ctx.save_for_backward(out, den, means, conics, colors, radii, op, rec, index.gids,
                              index.offsets, index.status)
        return out

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_out):
        n, H, W, normalize, eps, ts, tail, has_op, det, cull, cutoff = ctx.meta
        need = ctx.needs_input_grad
        if not (need[0] or need[1] or need[2] or need[4]) or n == 0:
            return (None,) * 14
        saved = ctx.saved_tensors
        out, den, means, conics, colors, radii, op = saved[:7]
        grad_out = grad_out.contiguous().to(torch.float32)
        dev = grad_out.device
        plan = ctx.plan
        if plan is not None and plan.generation == ctx.generation:
            if plan.moments_used:  # a second backward of the same forward
                plan.bwd_ws.zero_()
            plan.moments_used = True
            stream = _stream()
            _native.call("ss_render_backward_moments", _p(grad_out), None, _p(plan.records), n,
                         _p(den), _p(out), _p(plan.gids), plan.capacity, _p(plan.offsets), H, W,
                         ts, int(normalize), float(eps), float(tail), 0, _p(plan.bwd_ws),
                         plan.bwd_ws_bytes, _p(plan.status), stream)
            flat = torch.empty(9 * n, device=dev, dtype=torch.float32)
            g_means, g_conics = flat[:2 * n].view(n, 2), flat[2 * n:5 * n].view(n, 3)
            g_colors = flat[5 * n:8 * n].view(n, 3)
            g_opac = flat[8 * n:] if has_op else None
            _native.call("ss_render_backward_finalize", _p(plan.records), n, _p(plan.gids),
                         plan.capacity, _p(plan.offsets), H, W, ts, int(has_op), 0,
                         _p(plan.bwd_ws), _p(g_means), _p(g_conics), _p(g_colors), _p(g_opac),
                         stream)
        else:
            if plan is not None:  # the plan moved on to a later forward: rebuild this one's
                rec = pack_records(means, conics, colors, radii, op, H, W)
                index = index_from_records(rec, n, H, W, ts, cull, cutoff, exact=True)
            else:
                rec, gids, offsets, status = saved[7:]
                index = TileIndex(gids, offsets, ts, status)
            g_means, g_conics, g_colors, g_opac = _backward(
                grad_out, rec, n, den, out, index, H, W, normalize, eps, tail, has_op, det, dev)
        return (g_means if need[0] else None, g_conics if need[1] else None,
                g_colors if need[2] else None, None,
                g_opac if (has_op and need[4]) else None) + (None,) * 9


RENDER_TILE = 32  # default render tile (16 is also supported; the forward is identical)


def render_b200(means, conics, colors, radii, H: int, W: int, opacities=None,
                normalize: bool = True, eps: float = DEFAULT_EPS, tile_size: int = RENDER_TILE,
                support_fade: bool = False, sigma_cutoff: float = 3.0,
                support_fade_alpha: float | None = None, tile_ellipse_cull: bool = True,
                deterministic: bool = False):
    """Render with the reference's exact normalized / additive equations on the B200 library.

    Arguments mirror ``render_cuda_exact``; ``tile_size`` may be 16 (the reference default) or
    32 — every pixel still sums its Gaussians in ascending id, so the image is the same.
    ``tile_ellipse_cull`` only takes effect with the full support fade, the one case where
    culled pairs have exactly zero weight.
    ``deterministic`` selects the two-pass backward whose gradients are bitwise reproducible.
    """
    _check_cuda_f32(means, conics, colors)
    _check_shapes(means, conics, colors, radii, opacities)
    tile_grid(H, W, tile_size)
    if tile_size not in (16, 32):
        raise ValueError(f"render tile_size must be 16 or 32, got {tile_size}")
    if normalize:
        eps = validate_eps(eps)
    alpha = resolve_fade_alpha(support_fade, support_fade_alpha)
    tail = fade_tail(sigma_cutoff, alpha)
    cull = bool(tile_ellipse_cull) and alpha >= 1.0
    if opacities is not None and opacities.numel() == 0:
        opacities = None
    if opacities is not None and opacities.dtype != torch.float32:
        raise RuntimeError("StructSplat B200 renderer supports float32 tensors only.")
    return _B200Render.apply(means, conics, colors, radii, opacities, int(H), int(W),
                             bool(normalize), float(eps), int(tile_size), tail, cull,
                             float(sigma_cutoff), bool(deterministic))


def render_field(means, conics, colors, radii, H: int, W: int, chunk: int = 4096,
                 mode: str = "b200", opacities=None, scales=None, rotations=None,
                 support_fade: bool = False, sigma_cutoff: float = 3.0, color_grads=None,
                 support_fade_alpha: float | None = None, checkpoint_chunks: bool = False,
                 normalization_eps: float = DEFAULT_EPS, deterministic: bool = False):
    """``render_field`` with the reference's signature (render.py:319-414) on the B200 library.

    Every normalized mode (``b200``, ``normalized``, ``cuda``, ``cuda_tiled`` …) and every
    additive mode (``b200_additive``, ``additive``, ``cuda_additive`` …) evaluates the same
    equation as the reference; ``chunk`` and ``checkpoint_chunks`` are memory knobs of the
    reference's torch loop and have no effect here.  CUDA tensors only.
    """
    del chunk, checkpoint_chunks, scales, rotations
    if color_grads is not None:
        raise NotImplementedError(
            "affine colour gradients (color_grads) are not implemented by the B200 renderer")
    if mode in NORMALIZED_MODES:
        normalize = True
        eps = validate_eps(normalization_eps)
    elif mode in ADDITIVE_MODES:
        normalize = False
        eps = DEFAULT_EPS
    else:
        raise ValueError(
            f"unknown renderer {mode!r}; expected one of {NORMALIZED_MODES + ADDITIVE_MODES}")
    return render_b200(means, conics, colors, radii, H, W, opacities=opacities,
                       normalize=normalize, eps=eps, support_fade=support_fade,
                       sigma_cutoff=sigma_cutoff, support_fade_alpha=support_fade_alpha,
                       deterministic=deterministic)


# ---------------------------------------------------------------- passes reusing the pair loop

def gaussian_activity(means, conics, radii, H: int, W: int, chunk: int = 4096,
                      support_fade: bool = False, sigma_cutoff: float = 3.0,
                      support_fade_alpha: float | None = None) -> torch.Tensor:
    """Each Gaussian's summed unnormalised weight over the image (render.py:417-442).

    Opacity-free, like the reference's pruning helper; ``chunk`` is accepted for signature
    compatibility (there is no chunking here).  Deterministic.
    """
    del chunk
    if not means.is_cuda:
        raise RuntimeError("StructSplat B200 renderer requires CUDA tensors; pass device='cuda'.")
    n = means.shape[0]
    alpha = resolve_fade_alpha(support_fade, support_fade_alpha)
    tail = fade_tail(sigma_cutoff, alpha)
    means = means.detach().contiguous().to(torch.float32)
    conics = conics.detach().contiguous().to(torch.float32)
    rec = pack_records(means, conics, conics, radii.contiguous(), None, H, W)
    act = torch.empty(n, device=means.device, dtype=torch.float32)
    if n:
        r = radii.detach()
        mean_side = float((2 * r + 1).to(torch.float32).mean()) if n else 0.0
        lanes = 8 if mean_side * mean_side <= 96 else 32
        _native.call("ss_gaussian_activity", _p(rec), n, float(tail), lanes, _p(act), _stream())
    return act


@torch.no_grad()
def render_cuda_exact_with_coverage(means, conics, colors, radii, H: int, W: int,
                                    opacities=None, eps: float = DEFAULT_EPS,
                                    support_fade: bool = False, sigma_cutoff: float = 3.0,
                                    tile_size: int = RENDER_TILE):
    """Normalized RGB and the raw coverage (opacity-weighted weight sum, no ε) from one
    forward (cuda_render.py:229-253); inference only."""
    if not means.is_cuda:
        raise RuntimeError("joint CUDA rendering requires CUDA tensors")
    if any(t.dtype != torch.float32 for t in (means, conics, colors)):
        raise RuntimeError("joint CUDA rendering requires float32 tensors")
    eps = validate_eps(eps)
    _check_shapes(means, conics, colors, radii, opacities)
    if opacities is not None and opacities.numel() == 0:
        opacities = None
    n = means.shape[0]
    alpha = resolve_fade_alpha(support_fade, None)
    tail = fade_tail(sigma_cutoff, alpha)
    rec = pack_records(means.contiguous(), conics.contiguous(), colors.contiguous(),
                       radii.contiguous(), None if opacities is None else opacities.contiguous(),
                       H, W)
    index = index_from_records(rec, n, H, W, tile_size, alpha >= 1.0, sigma_cutoff)
    return _forward(rec, n, index, H, W, True, eps, tail, means.device)


class _RawWeightMap(Function):
    """den(p) = Σ_i o_i · visible_weight_i(p) over each Gaussian's clipped support, flattened to
    (H·W,), differentiable w.r.t. means, conics and opacities (fit.py:338-367)."""

    @staticmethod
    def forward(ctx, means, conics, radii, opacities, H, W, tail, cull, sigma_cutoff, tile_size):
        n = means.shape[0]
        means, conics = means.contiguous(), conics.contiguous()
        has_op = opacities is not None
        rec = pack_records(means, conics, conics, radii.contiguous(),
                           opacities.contiguous() if has_op else None, H, W)
        index = index_from_records(rec, n, H, W, tile_size, cull, sigma_cutoff)
        _, den = _forward(rec, n, index, H, W, False, 1.0, tail, means.device)
        ctx.save_for_backward(rec, index.gids, index.offsets, index.status)
        ctx.meta = (n, H, W, tile_size, tail, has_op)
        return den.view(-1)

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_den):
        rec, gids, offsets, status = ctx.saved_tensors
        n, H, W, ts, tail, has_op = ctx.meta
        if n == 0 or H * W == 0:
            return (None,) * 10
        dev = grad_den.device
        pixel_grad = torch.zeros(H * W, 4, device=dev, dtype=torch.float32)
        pixel_grad[:, 3] = grad_den.reshape(-1).to(torch.float32)
        cap = int(gids.numel())
        ws_bytes = _native.size_query("ss_render_backward_workspace_bytes", n, cap, H, W, 0)
        ws = torch.zeros(max(ws_bytes // 4, 4), device=dev, dtype=torch.float32)
        _native.call("ss_render_backward_moments", None, _p(pixel_grad), _p(rec), n, None, None,
                     _p(gids), cap, _p(offsets), H, W, ts, 0, 1.0, float(tail), 0, _p(ws),
                     ws_bytes, _p(status), _stream())
        g_means = torch.empty(n, 2, device=dev)
        g_conics = torch.empty(n, 3, device=dev)
        g_colors = torch.empty(n, 3, device=dev)
        g_opac = torch.empty(n, device=dev) if has_op else None
        _native.call("ss_render_backward_finalize", _p(rec), n, _p(gids), cap, _p(offsets), H, W,
                     ts, int(has_op), 0, _p(ws), _p(g_means), _p(g_conics), _p(g_colors),
                     _p(g_opac), _stream())
        need = ctx.needs_input_grad
        return (g_means if need[0] else None, g_conics if need[1] else None, None,
                g_opac if (has_op and need[3]) else None) + (None,) * 6


def raw_weight_map(means, conics, radii, H: int, W: int, opacities=None,
                   sigma_cutoff: float = 3.0, support_fade: bool = False,
                   support_fade_alpha: float | None = None, tile_size: int = RENDER_TILE):
    """Differentiable (H·W,) raw opacity-weighted weight sum Σ_i o_i G_i(p) — the accumulation
    behind the reference's mask and coverage losses (``_raw_weight_map_field``, fit.py:338-367),
    with the renderer's support window and fade."""
    _check_cuda_f32(means, conics, conics)
    if opacities is not None and opacities.numel() == 0:
        opacities = None
    alpha = resolve_fade_alpha(support_fade, support_fade_alpha)
    tail = fade_tail(sigma_cutoff, alpha)
    return _RawWeightMap.apply(means, conics, radii, opacities, int(H), int(W), tail,
                               alpha >= 1.0, float(sigma_cutoff), int(tile_size))
