"""Tile binning on the GPU is bit-exact against the reference's per-tile sets.

Offsets must be equal and every tile must list exactly the reference's Gaussians
(tests/test_render.py:376-414 of the reference); the library additionally lists them in
ascending id, so whole arrays are compared.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import cuda, require_cuda
from oracle import c_oracle, field_ref
from structsplat_b200 import render as R
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu


def _index(means, radii, H, W, ts, conics=None, cull=False, cutoff=3.0):
    m = cuda(means, torch.float32)
    r = cuda(radii, torch.int64)
    c = torch.zeros(m.shape[0], 3, device="cuda") if conics is None else cuda(conics, torch.float32)
    gids, offsets = R.build_tile_index(m, c, r, H, W, ts, ellipse_cull=cull, sigma_cutoff=cutoff)
    torch.cuda.synchronize()
    assert gids.dtype == torch.int32 and offsets.dtype == torch.int32
    return gids.cpu().numpy().astype(np.int64), offsets.cpu().numpy().astype(np.int64)


@pytest.mark.parametrize("name", golden_names("tile_"))
def test_tile_index_matches_reference_vectors(name):
    require_cuda()
    z = golden(name)
    gids, offsets = _index(z["means"], z["radii"], int(z["H"]), int(z["W"]), int(z["tile_size"]))
    assert np.array_equal(offsets, z["offsets"])
    assert np.array_equal(gids, z["gids_sorted"])


def test_known_answer_vector():
    require_cuda()
    gids, offsets = _index([[2.0, 2.0], [20.0, 20.0]], [[1, 1], [1, 1]], 8, 8, 4)
    assert offsets.tolist() == [0, 1, 1, 1, 1]
    assert gids.tolist() == [0]


@pytest.mark.parametrize("ts", [1, 4, 8, 16, 32])
@pytest.mark.parametrize("seed", [0, 1])
def test_random_fields_match_oracle(ts, seed):
    """Heavy-tailed scales (rectangles from one pixel to the whole image), centres off-image,
    non-finite and huge centres, ragged image sizes."""
    require_cuda()
    rng = np.random.default_rng(seed)
    H, W = int(rng.integers(17, 140)), int(rng.integers(17, 140))
    f = make_field(H, W, 700, seed=seed, log_sigma_std=1.2)
    means = f.means.copy()
    means[:40] = rng.uniform(-60, max(H, W) + 60, (40, 2))
    means[40] = [np.nan, 3.0]
    means[41] = [np.inf, 5.0]
    means[42] = [1e12, -1e12]
    means[43] = [2.5, 3.5]
    radii = field_ref.radii(torch.tensor(f.log_scales), torch.tensor(f.rotations), 3.0).numpy()
    radii[44] = [0, 0]
    radii[45] = [1 << 35, 2]
    gids, offsets = _index(means, radii, H, W, ts)
    ref_g, ref_o = c_oracle.tile_index(means, radii, H, W, ts)
    assert np.array_equal(offsets, ref_o)
    assert np.array_equal(gids, ref_g)
    assert not np.isin([40, 41, 42], gids).any()


@pytest.mark.parametrize("H, W", [(1, 1), (31, 33), (63, 65), (64, 64), (127, 129), (128, 128)])
def test_scan_regimes_match_oracle(H, W):
    """Tile sets on both sides of each scan regime's limit (one-pixel tiles, so T = H W): the
    count kernel's last CTA scans up to 4,095 tiles, the single-CTA scan kernel up to 16,383,
    CUB's device scan beyond."""
    require_cuda()
    f = make_field(H, W, 500, seed=H + W, log_sigma_std=0.6)
    radii = field_ref.radii(torch.tensor(f.log_scales), torch.tensor(f.rotations), 3.0).numpy()
    for _ in range(2):  # built twice: the same index both times
        gids, offsets = _index(f.means, radii, H, W, 1)
    ref_g, ref_o = c_oracle.tile_index(f.means, radii, H, W, 1)
    assert np.array_equal(offsets, ref_o)
    assert np.array_equal(gids, ref_g)


@pytest.mark.parametrize("n", [1024, 1025, 2048, 2049, 3072, 3073, 4096, 4097, 16384, 16385])
def test_single_tile_list_lengths(n):
    """One 16x16 tile that every Gaussian covers: its list is exactly ids 0 .. n-1, whichever
    sort a list of that length takes (the per-warp register sort up to 1,024 ids, the block
    radix sort with 2, 3 or 4 keys per thread up to 2,048 / 3,072 / 4,096, the shared-memory
    bitonic sort up to 16,384, the in-place one beyond), from the fill's arbitrary order."""
    require_cuda()
    rng = np.random.default_rng(n)
    means = rng.uniform(0, 16, (n, 2)).astype(np.float32)
    radii = rng.integers(1, 8, (n, 2))
    gids, offsets = _index(means, radii, 16, 16, 16)
    assert np.array_equal(offsets, [0, n])
    assert np.array_equal(gids, np.arange(n))


@pytest.mark.parametrize("n", [3000, 20000])
def test_long_tile_lists_are_sorted(n):
    """Lists longer than the per-warp sort (1024) and the per-CTA shared-memory sort (16384)."""
    require_cuda()
    rng = np.random.default_rng(5)
    H = W = 48
    means = rng.uniform(16, 32, (n, 2)).astype(np.float32)
    radii = rng.integers(1, 20, (n, 2))
    gids, offsets = _index(means, radii, H, W, 16)
    ref_g, ref_o = c_oracle.tile_index(means, radii, H, W, 16)
    assert (np.diff(ref_o) > 1024).any()
    assert np.array_equal(offsets, ref_o)
    assert np.array_equal(gids, ref_g)


def test_ellipse_cull_only_drops_zero_weight_pairs():
    """With the cull the lists shrink but stay a superset of every pair with faded weight."""
    require_cuda()
    rng = np.random.default_rng(22)
    N, H, W = 200, 96, 100
    means = np.stack([rng.uniform(-3, W + 3, N), rng.uniform(-3, H + 3, N)], 1).astype(np.float32)
    ls = np.log(np.stack([np.exp(rng.uniform(np.log(2), np.log(12), N)),
                          np.exp(rng.uniform(np.log(0.5), np.log(1.2), N))], 1)).astype(np.float32)
    rot = rng.uniform(0, np.pi, N).astype(np.float32)
    conics = field_ref.conics(torch.tensor(ls), torch.tensor(rot)).numpy()
    radii = field_ref.radii(torch.tensor(ls), torch.tensor(rot), 3.0).numpy()
    full_g, full_o = _index(means, radii, H, W, 16, conics)
    cull_g, cull_o = _index(means, radii, H, W, 16, conics, cull=True)
    assert cull_o[-1] < full_o[-1]
    for t in range(len(full_o) - 1):
        assert set(cull_g[cull_o[t]:cull_o[t + 1]]) <= set(full_g[full_o[t]:full_o[t + 1]])


def test_empty_inputs():
    require_cuda()
    gids, offsets = _index(np.zeros((0, 2), np.float32), np.zeros((0, 2), np.int64), 20, 30, 16)
    assert gids.size == 0 and offsets.tolist() == [0] * 5
    gids, offsets = _index([[5.0, 5.0]], [[2, 2]], 0, 30, 16)
    assert gids.size == 0 and offsets.tolist() == [0]
