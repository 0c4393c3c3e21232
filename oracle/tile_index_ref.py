"""CPU oracle of the tile → Gaussian index (test infrastructure only).

Restates ``_build_tile_index`` (``src/structsplat/cuda_render.py:177-226``): every Gaussian
with a non-empty clipped support rectangle is listed in each ``tile_size``² tile its rectangle
touches; ``offsets`` (T+1) delimits each tile's list.  The reference's within-tile order is
not part of its contract (``tests/test_render.py:401-409``: offsets equal, per-tile sets
equal); this oracle lists each tile's Gaussians in ascending id, the order the CUDA
library produces.
"""
from __future__ import annotations

import numpy as np

from .render_ref import support_rect


def tile_grid(H: int, W: int, tile_size: int):
    if tile_size <= 0 or tile_size * tile_size > 1024:
        raise ValueError("tile_size must be positive with tile_size^2 <= 1024")
    tiles_x = (W + tile_size - 1) // tile_size
    tiles_y = (H + tile_size - 1) // tile_size
    return tiles_x, tiles_y


def build_tile_index(means, radii, H: int, W: int, tile_size: int):
    """Return ``(gids int64 [entries], offsets int64 [T+1])`` with ascending ids per tile."""
    tiles_x, tiles_y = tile_grid(H, W, tile_size)
    num_tiles = tiles_x * tiles_y
    x0, y0, tx, ty = (t.numpy() for t in support_rect(means, radii, H, W))
    live = np.nonzero((tx > 0) & (ty > 0))[0]
    if num_tiles == 0 or live.size == 0:
        return np.zeros(0, np.int64), np.zeros(num_tiles + 1, np.int64)
    ts = tile_size
    gx0 = x0[live] // ts
    gy0 = y0[live] // ts
    gx1 = (x0[live] + tx[live] - 1) // ts
    gy1 = (y0[live] + ty[live] - 1) // ts
    gw = gx1 - gx0 + 1
    cnt = gw * (gy1 - gy0 + 1)
    owner = np.repeat(live, cnt)
    first = np.cumsum(cnt) - cnt
    k = np.arange(owner.size) - np.repeat(first, cnt)
    gwr = np.repeat(gw, cnt)
    tile = (np.repeat(gy0, cnt) + k // gwr) * tiles_x + (np.repeat(gx0, cnt) + k % gwr)
    order = np.lexsort((owner, tile))      # by tile, then by Gaussian id
    per_tile = np.bincount(tile, minlength=num_tiles)
    offsets = np.zeros(num_tiles + 1, np.int64)
    np.cumsum(per_tile, out=offsets[1:])
    return owner[order].astype(np.int64), offsets


def tile_sets(gids, offsets):
    """Per-tile sorted id lists — the order-free form the reference's tests compare."""
    gids = np.asarray(gids)
    offsets = np.asarray(offsets)
    return [sorted(gids[offsets[t]:offsets[t + 1]].tolist()) for t in range(len(offsets) - 1)]
