"""One image across ranks in bands of tile rows: the forward is independent per band, the
backward's parameter gradients are summed over the bands with one all-reduce.

A band is the tile rows [t0, t1) of the image (pixel rows [y0, y1), y0 = t0 * tile size).  Every
rank projects and bins the whole field for the whole image (O(N + entries), a small part of a
step), then renders and differentiates only its band's tiles: the band is described to the
library as a one-image batch whose tiles are the window [t0, t1) of the image's tile rows
(``first_tile = -t0 * tiles_x``, the tile offsets taken from row t0), so its pixels use the
full image's records, tile lists and per-pixel evaluation and the band images stack into the
full image bitwise.  The gradients w.r.t. the RS parameters are linear in the backward's
per-Gaussian moments, which are sums over pixels, so the sum of the bands' gradients is the
full image's gradient (to float rounding of the sum); that sum is the one exchange step, an
all-reduce of 9 N floats (means 2, log-scales 2, rotation 1, colours 3, opacity logit 1).
"""
from __future__ import annotations

import ctypes

import torch

from . import _native
from .fit import RenderPlan
from .render import RENDER_TILE, _p, _stream, tile_grid

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
    """Forward + backward of the band [y0, y1) of an H×W image: the full image's projection and
    tile index (a RenderPlan), rendered and differentiated over the band's tiles only."""

    def __init__(self, params: dict, H: int, W: int, y0: int, y1: int, **plan_kw):
        if not 0 <= y0 <= y1 <= H:
            raise ValueError(f"band rows [{y0}, {y1}) outside the image of height {H}")
        ts = plan_kw.get("tile_size", RENDER_TILE)
        if y0 % ts:
            raise ValueError(f"band start {y0} is not a multiple of the tile size {ts}")
        if y1 % ts and y1 != H:
            raise ValueError(f"band end {y1} is neither a multiple of the tile size nor H")
        self.H, self.W, self.y0, self.y1, self.ts = H, W, y0, y1, ts
        self.plan = RenderPlan.for_field(params, H, W, **plan_kw)
        self.n = n = params["means"].shape[0]
        dev = params["means"].device
        tiles_x, _ = tile_grid(H, W, ts)
        self.t0 = y0 // ts
        self.band_tiles = ((y1 - y0 + ts - 1) // ts) * tiles_x
        self._tables = {
            "image": torch.tensor([[H, W, tiles_x, -self.t0 * tiles_x]], dtype=torch.int32,
                                  device=dev),
            "pixel_base": torch.zeros(1, dtype=torch.int64, device=dev),
            "gaussian_base": torch.tensor([0, n], dtype=torch.int32, device=dev),
            "gaussian_image": torch.zeros(max(n, 1), dtype=torch.int32, device=dev),
            "tile_image": torch.zeros(max(self.band_tiles, 1), dtype=torch.int32, device=dev),
        }
        t = self._tables
        self.batch = _native.SsBatch(
            images=1, tile_size=ts, tiles=self.band_tiles, pixels=H * W,
            image_table=t["image"].data_ptr(), pixel_base=t["pixel_base"].data_ptr(),
            gaussian_base=t["gaussian_base"].data_ptr(),
            gaussian_image=t["gaussian_image"].data_ptr() if n else None,
            tile_image=t["tile_image"].data_ptr())
        self.ref = ctypes.byref(self.batch)
        f32 = dict(device=dev, dtype=torch.float32)
        self.image = torch.zeros(H, W, 3, **f32)
        self.den = torch.zeros(H, W, **f32)
        p = self.plan
        self.g = {"means": torch.zeros(n, 2, **f32), "conics": torch.zeros(n, 3, **f32),
                  "colors": torch.zeros(n, 3, **f32), "opacities": torch.zeros(n, **f32),
                  "log_scales": torch.zeros(n, 2, **f32), "rotations": torch.zeros(n, **f32),
                  "opacity_logits": torch.zeros(n, **f32)}
        self.ws_bytes = _native.size_query("ss_render_backward_workspace_bytes", n, p.capacity,
                                           H, W, int(p.deterministic))
        self.ws = torch.zeros(max(self.ws_bytes // 4, 4), **f32)

    def _offsets(self):
        tiles_x, _ = tile_grid(self.H, self.W, self.ts)
        return ctypes.c_void_p(self.plan.offsets.data_ptr() + 4 * self.t0 * tiles_x)

    def forward_backward(self, params: dict, grad_out: torch.Tensor):
        """Band image (y1-y0, W, 3) and the band's gradients w.r.t. the RS parameters, given the
        full image's grad_out (H, W, 3)."""
        n, p = self.n, self.plan
        if self.y1 == self.y0 or n == 0:
            z = {k: torch.zeros_like(params[k]) for k in GRAD_NAMES if params.get(k) is not None}
            return self.image[self.y0:self.y1], z
        p.project_count(params)
        p.fill()
        offsets = self._offsets()
        _native.call("ss_batch_render_forward", self.ref, _p(p.records), n, _p(p.gids),
                     p.capacity, offsets, int(p.normalize), float(p.eps), float(p.tail),
                     _p(self.image), _p(self.den), _p(p.status), _stream())
        go = grad_out.contiguous()
        g = self.g
        has_op = p.has_opacity
        _native.call("ss_batch_render_backward", self.ref, _p(go), _p(p.records), n,
                     _p(self.den), _p(self.image), _p(p.gids), p.capacity, offsets,
                     int(p.normalize), float(p.eps), float(p.tail), int(has_op),
                     _p(g["means"]), _p(g["conics"]), _p(g["colors"]),
                     _p(g["opacities"]) if has_op else None, int(p.deterministic), _p(self.ws),
                     self.ws_bytes, _p(p.status), _stream())
        logits = params.get("opacity_logits") if has_op else None
        _native.call("ss_project_rs_backward", _p(params["log_scales"]), _p(params["rotations"]),
                     _p(logits), n, float(p.dilation), _p(g["conics"]),
                     _p(g["opacities"]) if has_op else None, _p(g["log_scales"]),
                     _p(g["rotations"]), _p(g["opacity_logits"]) if has_op else None, _stream())
        grads = {"means": g["means"], "log_scales": g["log_scales"],
                 "rotations": g["rotations"], "colors": g["colors"]}
        if has_op:
            grads["opacity_logits"] = g["opacity_logits"]
        return self.image[self.y0:self.y1], grads


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
