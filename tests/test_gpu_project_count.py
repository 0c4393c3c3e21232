"""The fused projection + tile count (``ss_project_rs_index_count`` and its batch form) against
``ss_project_rs`` followed by ``ss_tile_index_count``: the records and the offsets are bitwise
equal, with and without the ellipse cull, for tile sets on both sides of the count kernel's
own scan (up to 4,095 tiles) and beyond it, for an empty field and for an empty image; the
region the call is asked to clear is zeroed, and nothing past it."""
from __future__ import annotations

import pytest
import torch

from gpu_helpers import require_cuda
from structsplat_b200 import _native
from structsplat_b200.batch import Batch, PARAM_NAMES
from structsplat_b200.render import RECORD_FLOATS, _p, _stream
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu


def _field(H, W, n, seed):
    f = make_field(max(H, 1), max(W, 1), n, seed=seed, log_sigma_std=0.8)
    return {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}


def _bufs(n, T, wsb):
    rec = torch.full((max(n, 1) * RECORD_FLOATS,), -7.0, device="cuda")
    off = torch.full((T + 1,), -1, dtype=torch.int32, device="cuda")
    ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    return rec, off, ws, status


def _rs(p):
    return (_p(p["means"]), _p(p["log_scales"]), _p(p["rotations"]), _p(p["colors"]),
            _p(p["opacity_logits"]))


@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("H, W, ts, n", [
    (96, 80, 16, 700),     # 30 tiles
    (1024, 1000, 16, 900),  # 4,032 tiles: the count kernel's own scan, four rounds
    (1024, 1024, 16, 900),  # 4,096 tiles: the scan kernel
    (300, 200, 1, 400),     # 60,000 tiles: CUB's scan
    (50, 60, 32, 0),        # no Gaussians
    (0, 40, 16, 30),        # an empty image: the records are still written
])
def test_fused_project_count_matches_the_two_calls(H, W, ts, n, cull):
    require_cuda()
    p = _field(H, W, n, seed=H + W + n)
    T = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
    wsb = _native.size_query("ss_tile_index_workspace_bytes", n, H, W, ts)
    r1, o1, w1, s1 = _bufs(n, T, wsb)
    r2, o2, w2, s2 = _bufs(n, T, wsb)
    _native.call("ss_project_rs", *_rs(p), n, 0.25, 3.0, H, W, _p(r1), None, None, _stream())
    _native.call("ss_tile_index_count", _p(r1), n, H, W, ts, cull, 3.0, _p(o1), _p(w1), wsb,
                 _p(s1), _stream())
    for _ in range(2):  # twice over the same workspace: the same offsets
        clear = torch.full((4096,), 7, dtype=torch.uint8, device="cuda")
        _native.call("ss_project_rs_index_count", *_rs(p), n, 0.25, 3.0, H, W, ts, cull, _p(r2),
                     _p(o2), _p(w2), wsb, _p(clear), 4096 - 16, _p(s2), _stream())
        assert not clear[:4096 - 16].any() and bool((clear[4096 - 16:] == 7).all())
    torch.cuda.synchronize()
    assert torch.equal(r1[: n * RECORD_FLOATS].view(torch.int32),
                       r2[: n * RECORD_FLOATS].view(torch.int32))
    assert torch.equal(o1, o2)
    assert int(s1.item()) == int(s2.item()) == 0


def test_batch_fused_project_count_matches_the_two_calls():
    require_cuda()
    sizes, counts = [(64, 96), (37, 50), (1, 1), (128, 128), (40, 33)], [500, 120, 3, 1500, 0]
    fields = [_field(H, W, n, seed=b) for b, ((H, W), n) in enumerate(zip(sizes, counts))]
    batch = Batch(sizes, counts)
    p = Batch.concat_fields(fields)
    n = batch.n
    wsb = _native.size_query("ss_batch_tile_index_workspace_bytes", batch.ref, n)
    r1, o1, w1, s1 = _bufs(n, batch.tiles, wsb)
    r2, o2, w2, s2 = _bufs(n, batch.tiles, wsb)
    _native.call("ss_batch_project_rs", batch.ref, *_rs(p), n, 0.0, 3.0, _p(r1), _stream())
    _native.call("ss_batch_tile_index_count", batch.ref, _p(r1), n, 1, 3.0, _p(o1), _p(w1), wsb,
                 _p(s1), _stream())
    _native.call("ss_batch_project_rs_index_count", batch.ref, *_rs(p), n, 0.0, 3.0, 1, _p(r2),
                 _p(o2), _p(w2), wsb, None, 0, _p(s2), _stream())
    torch.cuda.synchronize()
    assert torch.equal(r1.view(torch.int32), r2.view(torch.int32))
    assert torch.equal(o1, o2)
