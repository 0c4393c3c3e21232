"""One image split into bands of tile rows across two gloo ranks on the CPU (the oracle stands in
for each rank's band: the full image's pixels of the band rows, and the gradients of those
pixels alone): the band images stack into the full image and the all-reduced band gradients
are the full image's gradients."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from oracle import field_ref, render_ref
from structsplat_b200.bands import all_reduce_grads, band_rows
from structsplat_b200.synthetic import make_field

H, W, N, TS = 70, 52, 160, 16


def _inputs():
    f = make_field(H, W, N, seed=9)
    ls, rot = torch.tensor(f.log_scales), torch.tensor(f.rotations)
    means = torch.tensor(f.means, dtype=torch.float64)
    conics = field_ref.conics(ls, rot).double()
    radii = field_ref.radii(ls, rot, 3.0)
    colors = torch.tensor(f.colors, dtype=torch.float64)
    opac = torch.sigmoid(torch.tensor(f.opacity_logits, dtype=torch.float64))
    g = torch.Generator().manual_seed(3)
    grad_out = torch.randn(H, W, 3, generator=g, dtype=torch.float64)
    return means, conics, colors, radii, opac, grad_out


def _band(rank, world):
    """A rank's band as the library computes it: the full image's records and tile lists,
    rendered and differentiated over the band's rows only."""
    means, conics, colors, radii, opac, grad_out = _inputs()
    y0, y1 = band_rows(H, W, rank, world, TS)
    band_grad = torch.zeros_like(grad_out)
    band_grad[y0:y1] = grad_out[y0:y1]
    img, _, grads = render_ref.render_with_grads(means, conics, colors, radii, H, W, band_grad,
                                                 opacities=opac)
    return (y0, y1), img[y0:y1], grads


def test_bands_cover_the_tile_rows():
    for world in (1, 2, 3, 5, 8):
        rows = [band_rows(H, W, r, world, TS) for r in range(world)]
        assert rows[0][0] == 0 and rows[-1][1] == H
        for (a0, a1), (b0, b1) in zip(rows, rows[1:]):
            assert a1 == b0 and a0 % TS == 0
    with pytest.raises(ValueError):
        band_rows(H, W, 2, 2, TS)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=__import__("datetime").timedelta(seconds=60))
    try:
        rows, img, grads = _band(rank, world)
        total = all_reduce_grads(grads)
        out.put((rank, rows, img.numpy(), {k: v.numpy() for k, v in total.items()}))
    finally:
        torch.distributed.destroy_process_group()


def test_two_gloo_ranks_sum_band_gradients_to_the_full_image():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    means, conics, colors, radii, opac, grad_out = _inputs()
    img, _, want = render_ref.render_with_grads(means, conics, colors, radii, H, W, grad_out,
                                                opacities=opac)
    stacked = np.concatenate([g[2] for g in got], axis=0)
    assert np.array_equal(stacked, img.numpy())
    for k in ("means", "conics", "colors", "opacities"):
        for _, _, _, total in got:
            ref = want[k].numpy()
            assert np.abs(total[k] - ref).max() <= 1e-9 * max(np.abs(ref).max(), 1.0), k
