"""One image across ranks in bands of tile rows: the forward is independent per band, the
backward's parameter gradients are summed over the bands with one all-reduce.

A band is the rows [y0, y1) of the image, y0 a multiple of the tile size, rendered as an image
of its own with the means shifted by -y0 (an integer: exact in float, so every Gaussian keeps
its rounded centre, support rectangle, tile lists and ellipse cull inside the band).  Pixels
of the band see exactly the Gaussians and arithmetic of the full image, so the band images
stack into the full image bitwise.  The gradients w.r.t. the RS parameters are linear in the
backward's per-Gaussian moments, which are sums over pixels, so the sum of the bands'
gradients is the full image's gradient (to float rounding of the sum); that sum is the one
exchange step, an all-reduce of 9 N floats (means 2, log-scales 2, rotation 1, colours 3,
opacity logit 1).
"""
from __future__ import annotations

import torch

from .fit import RenderPlan
from .render import RENDER_TILE, tile_grid

GRAD_NAMES = ("means", "log_scales", "rotations", "colors", "opacity_logits")


def band_rows(H: int, W: int, rank: int, world: int, tile_size: int = RENDER_TILE):
    """Rows [y0, y1) of rank ``rank``'s band: the tile rows split as evenly as possible (a rank
    may get an empty band when there are fewer tile rows than ranks)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} out of range for world size {world}")
    _, tiles_y = tile_grid(H, W, tile_size)
    t0, t1 = rank * tiles_y // world, (rank + 1) * tiles_y // world
    return min(t0 * tile_size, H), min(t1 * tile_size, H)


class BandPlan:
    """Forward + backward of one band of an H×W image (a RenderPlan of the band's rows)."""

    def __init__(self, params: dict, H: int, W: int, y0: int, y1: int, **plan_kw):
        if not 0 <= y0 <= y1 <= H:
            raise ValueError(f"band rows [{y0}, {y1}) outside the image of height {H}")
        ts = plan_kw.get("tile_size", RENDER_TILE)
        if y0 % ts:
            raise ValueError(f"band start {y0} is not a multiple of the tile size {ts}")
        self.H, self.W, self.y0, self.y1 = H, W, y0, y1
        self.shift = torch.tensor([0.0, float(y0)], device=params["means"].device)
        self.means = params["means"] - self.shift
        local = dict(params, means=self.means)
        self.plan = RenderPlan.for_field(local, max(y1 - y0, 0), W, **plan_kw) if y1 > y0 else None

    def forward_backward(self, params: dict, grad_out: torch.Tensor):
        """Band image (y1-y0, W, 3) and the band's gradients w.r.t. the RS parameters, given the
        full image's grad_out (H, W, 3)."""
        n = params["means"].shape[0]
        if self.plan is None:
            z = {k: torch.zeros_like(params[k]) for k in GRAD_NAMES if params.get(k) is not None}
            return params["means"].new_zeros(0, self.W, 3), z
        torch.sub(params["means"], self.shift, out=self.means)
        local = dict(params, means=self.means)
        g_band = grad_out[self.y0:self.y1].contiguous()
        grads = self.plan.forward_backward(local, g_band)
        image = self.plan.image.view(self.y1 - self.y0, self.W, 3)
        assert grads["means"].shape[0] == n
        return image, grads


def all_reduce_grads(grads: dict, group=None) -> dict:
    """Sum of every rank's band gradients (one all-reduce of the concatenated tensors, in
    sorted key order so every rank packs them alike: 9 N floats for the RS parameters); the
    gradients themselves when no process group is initialised."""
    names = sorted(k for k, v in grads.items() if v is not None)
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return {k: grads[k] for k in names}
    flat = torch.cat([grads[k].reshape(-1) for k in names])
    torch.distributed.all_reduce(flat, op=torch.distributed.ReduceOp.SUM, group=group)
    out, at = {}, 0
    for k in names:
        m = grads[k].numel()
        out[k] = flat[at:at + m].view_as(grads[k])
        at += m
    return out
