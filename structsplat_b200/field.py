"""Fit-path rendering straight from the RS field parameters.

``GaussianField.conics / radii / opacity_values`` (gaussians.py:270-321) are a chain of ~10
elementwise torch ops forward and ~20 backward per iteration.  Here one kernel projects the
field tensors (means, log_scales, rotations, colors, opacity logits — the reference's field
layout, gaussians.py:15-29) straight into the packed splat records, and the render backward is
followed by one kernel applying the chain rule back to log-scales, rotations and logits.
"""
from __future__ import annotations

import torch
from torch.autograd import Function
from torch.autograd.function import once_differentiable

from . import _native
from .render import (DEFAULT_EPS, EAGER_PLANS, RECORD_FLOATS, RENDER_TILE, TileIndex, _backward,
                     _forward, _p, _stream, fade_tail, index_from_records, resolve_fade_alpha,
                     tile_grid, validate_eps)


def project(means, log_scales, rotations, colors, opacity_logits, H: int, W: int,
            sigma_cutoff: float = 3.0, dilation: float = 0.0, want_conics: bool = False):
    """Splat records (and optionally conics (N,3) f32 / radii (N,2) int64) of an RS field."""
    if dilation < 0.0:
        raise ValueError(f"dilation must be >= 0, got {dilation}")
    n = means.shape[0]
    dev = means.device
    rec = torch.empty(max(n, 1) * RECORD_FLOATS, device=dev, dtype=torch.float32)
    conics = torch.empty(n, 3, device=dev, dtype=torch.float32) if want_conics else None
    radii = torch.empty(n, 2, device=dev, dtype=torch.int64) if want_conics else None
    if n:
        _native.call("ss_project_rs", _p(means), _p(log_scales), _p(rotations), _p(colors),
                     _p(opacity_logits), n, float(dilation), float(sigma_cutoff), H, W, _p(rec),
                     _p(conics), _p(radii), _stream())
    return rec, conics, radii


class _B200RenderRS(Function):
    @staticmethod
    def forward(ctx, means, log_scales, rotations, colors, logits, H, W, normalize, eps,
                tile_size, tail, cull, sigma_cutoff, dilation, deterministic):
        n = means.shape[0]
        means, log_scales = means.contiguous(), log_scales.contiguous()
        rotations, colors = rotations.contiguous(), colors.contiguous()
        logits = None if logits is None else logits.contiguous()
        ctx.meta = (n, H, W, bool(normalize), float(eps), int(tile_size), float(tail),
                    logits is not None, float(dilation), bool(deterministic), bool(cull),
                    float(sigma_cutoff))
        if not deterministic and n and H * W:
            # the fast path: the problem's buffers persist between calls (EagerPlan)
            plan = EAGER_PLANS.get(n, H, W, tile_size, cull, sigma_cutoff, means.device)
            stream = _stream()
            _native.call("ss_project_rs_index_count", _p(means), _p(log_scales), _p(rotations),
                         _p(colors), _p(logits), n, float(dilation), float(sigma_cutoff), H, W,
                         tile_size, int(cull), _p(plan.records), _p(plan.offsets),
                         _p(plan.idx_ws), plan.idx_ws_bytes, _p(plan.step_block),
                         plan.step_block.numel(), _p(plan.status), stream)
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
            ctx.save_for_backward(out, den, means, log_scales, rotations, colors, logits)
            return out
        rec, _, _ = project(means, log_scales, rotations, colors, logits, H, W, sigma_cutoff,
                            dilation)
        index = index_from_records(rec, n, H, W, tile_size, cull, sigma_cutoff,
                                   exact=bool(deterministic))
        out, den = _forward(rec, n, index, H, W, normalize, eps, tail, means.device)
        ctx.plan = None
        ctx.save_for_backward(out, den, means, log_scales, rotations, colors, logits, rec,
                              index.gids, index.offsets, index.status)
        return out

    @staticmethod
    @once_differentiable
    def backward(ctx, grad_out):
        n, H, W, normalize, eps, ts, tail, has_op, dilation, det, cull, cutoff = ctx.meta
        if n == 0:
            return (None,) * 15
        saved = ctx.saved_tensors
        out, den, means, log_scales, rotations, colors, logits = saved[:7]
        grad_out = grad_out.contiguous().to(torch.float32)
        need = ctx.needs_input_grad
        plan = ctx.plan
        if plan is not None and plan.generation == ctx.generation:
            dev = grad_out.device
            if plan.moments_used:  # a second backward of the same forward
                plan.bwd_ws.zero_()
            plan.moments_used = True
            stream = _stream()
            _native.call("ss_render_backward_moments", _p(grad_out), None, _p(plan.records), n,
                         _p(den), _p(out), _p(plan.gids), plan.capacity, _p(plan.offsets), H, W,
                         ts, int(normalize), float(eps), float(tail), 0, _p(plan.bwd_ws),
                         plan.bwd_ws_bytes, _p(plan.status), stream)
            flat = torch.empty(9 * n, device=dev, dtype=torch.float32)
            g_means, g_ls = flat[:2 * n].view(n, 2), flat[2 * n:4 * n].view(n, 2)
            g_rot, g_colors = flat[4 * n:5 * n], flat[5 * n:8 * n].view(n, 3)
            g_logits = flat[8 * n:] if has_op else None
            _native.call("ss_render_backward_finalize_rs", _p(plan.records), n, _p(plan.gids),
                         plan.capacity, _p(plan.offsets), H, W, ts, 0, _p(plan.bwd_ws),
                         _p(log_scales), _p(rotations), _p(logits), float(dilation),
                         _p(g_means), _p(g_ls), _p(g_rot), _p(g_colors), _p(g_logits),
                         stream)
        else:
            if plan is not None:  # the plan moved on to a later forward: rebuild this one's
                rec, _, _ = project(means, log_scales, rotations, colors, logits, H, W, cutoff,
                                    dilation)
                index = index_from_records(rec, n, H, W, ts, cull, cutoff, exact=True)
            else:
                rec, gids, offsets, status = saved[7:]
                index = TileIndex(gids, offsets, ts, status)
            g_means, g_conics, g_colors, g_opac = _backward(
                grad_out, rec, n, den, out, index, H, W, normalize, eps, tail, has_op, det,
                grad_out.device)
            g_ls = torch.empty_like(log_scales)
            g_rot = torch.empty_like(rotations)
            g_logits = torch.empty_like(logits) if has_op else None
            _native.call("ss_project_rs_backward", _p(log_scales), _p(rotations), _p(logits), n,
                         float(dilation), _p(g_conics), _p(g_opac), _p(g_ls), _p(g_rot),
                         _p(g_logits), _stream())
        return (g_means if need[0] else None, g_ls if need[1] else None,
                g_rot if need[2] else None, g_colors if need[3] else None,
                g_logits if (has_op and need[4]) else None) + (None,) * 10


def render_gaussians(means, log_scales, rotations, colors, H: int, W: int,
                     opacity_logits=None, normalize: bool = True, eps: float = DEFAULT_EPS,
                     sigma_cutoff: float = 3.0, dilation: float = 0.0,
                     support_fade: bool = False, support_fade_alpha: float | None = None,
                     tile_size: int = RENDER_TILE, tile_ellipse_cull: bool = True,
                     deterministic: bool = False):
    """Render an RS field; differentiable w.r.t. all five parameter tensors.

    Equivalent to ``render_field(f.means, f.conics(dilation), f.colors,
    f.radii(sigma_cutoff, dilation), H, W, opacities=f.opacity_values(), …)`` with the
    reference's ``GaussianField`` f.
    """
    if not means.is_cuda:
        raise RuntimeError("StructSplat B200 renderer requires CUDA tensors; pass device='cuda'.")
    for t in (means, log_scales, rotations, colors):
        if t.dtype != torch.float32:
            raise RuntimeError("StructSplat B200 renderer supports float32 tensors only.")
    n = means.shape[0]
    if log_scales.shape != (n, 2) or rotations.shape != (n,) or colors.shape != (n, 3):
        raise ValueError("field tensors must be means (N,2), log_scales (N,2), rotations (N,), "
                         "colors (N,3)")
    tile_grid(H, W, tile_size)
    if tile_size not in (16, 32):
        raise ValueError(f"render tile_size must be 16 or 32, got {tile_size}")
    if normalize:
        eps = validate_eps(eps)
    alpha = resolve_fade_alpha(support_fade, support_fade_alpha)
    tail = fade_tail(sigma_cutoff, alpha)
    cull = bool(tile_ellipse_cull) and alpha >= 1.0
    return _B200RenderRS.apply(means, log_scales, rotations, colors, opacity_logits, int(H),
                               int(W), bool(normalize), float(eps), int(tile_size), tail, cull,
                               float(sigma_cutoff), float(dilation), bool(deterministic))
