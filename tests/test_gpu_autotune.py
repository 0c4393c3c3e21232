"""The autotuner picks a launch shape by timing, caches it, and shapes never change results."""
from __future__ import annotations

import pytest
import torch

from gpu_helpers import require_cuda
from structsplat_b200 import _native, autotune
from structsplat_b200.batch import FitSettings, PARAM_NAMES, fit_batch
from structsplat_b200.fit import RenderPlan
from structsplat_b200.synthetic import make_field, make_target

pytestmark = pytest.mark.gpu


def _field(H, W, n, seed):
    f = make_field(H, W, n, seed=seed)
    return {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}


def test_backward_warps_do_not_change_deterministic_gradients():
    require_cuda()
    H, W = 160, 144
    params = _field(H, W, 3000, seed=1)
    go = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    for ts, choices in ((16, (4, 8)), (32, (8, 16))):
        grads = []
        for warps in choices:
            _native.call("ss_set_backward_warps", ts, warps)
            plan = RenderPlan.for_field(params, H, W, deterministic=True, tile_size=ts)
            grads.append({k: v.clone() for k, v in plan.forward_backward(params, go).items()})
        _native.call("ss_set_backward_warps", ts, 0)
        for k in grads[0]:
            assert torch.equal(grads[0][k], grads[1][k]), (ts, k)


def test_tune_render_picks_a_candidate_and_caches_it(tmp_path, monkeypatch):
    require_cuda()
    monkeypatch.setenv("STRUCTSPLAT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    H, W = 256, 256
    params = _field(H, W, 8000, seed=3)
    go = torch.randn(H, W, 3, device="cuda")
    r = autotune.tune_render(params, H, W, go, repeats=3)
    assert (r.tile_size, r.backward_warps) in autotune.CANDIDATES
    assert len(r.times_ms) == len(autotune.CANDIDATES) and not r.cached
    assert _native.lib().ss_get_backward_warps(r.tile_size) == r.backward_warps
    again = autotune.tune_render(params, H, W, go, repeats=3)
    assert again.cached and (again.tile_size, again.backward_warps) == (r.tile_size,
                                                                        r.backward_warps)
    for ts in (16, 32):
        _native.call("ss_set_backward_warps", ts, 0)


def test_tuned_batched_fit_reaches_the_same_psnr(tmp_path, monkeypatch):
    require_cuda()
    monkeypatch.setenv("STRUCTSPLAT_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    sizes = [(96, 128), (64, 64)]
    targets = [torch.tensor(make_target(h, w, seed=30 + b), device="cuda")
               for b, (h, w) in enumerate(sizes)]
    a = [_field(h, w, int(0.1 * h * w), seed=40 + b) for b, (h, w) in enumerate(sizes)]
    b = [{k: v.clone() for k, v in f.items()} for f in a]
    s = FitSettings()
    ha = fit_batch(a, targets, iters=30, settings=s, tune=True)
    hb = fit_batch(b, targets, iters=30, settings=s, tile_size=16)
    assert ha["tuned"] is not None
    for pa, pb in zip(ha["final_psnr"], hb["final_psnr"]):
        assert abs(pa - pb) <= 0.01
    for ts in (16, 32):
        _native.call("ss_set_backward_warps", ts, 0)


def test_dependent_launch_does_not_change_results():
    """The step's kernels give bitwise the same image and deterministic gradients whether or not
    they may start while their predecessor drains."""
    require_cuda()
    H, W = 160, 144
    params = _field(H, W, 3000, seed=4)
    go = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    runs = []
    for enable in (1, 0):
        _native.call("ss_set_dependent_launch", enable)
        try:
            plan = RenderPlan.for_field(params, H, W, deterministic=True)
            grads = {k: v.clone() for k, v in plan.forward_backward(params, go).items()}
            torch.cuda.synchronize()
            runs.append((plan.image.clone(), grads))
        finally:
            _native.call("ss_set_dependent_launch", 1)
    assert torch.equal(runs[0][0], runs[1][0])
    for k in runs[0][1]:
        assert torch.equal(runs[0][1][k], runs[1][1][k]), k


def test_forward_chunk_depth_does_not_change_the_image():
    """A streamed list (longer than the 512-record stage) renders bitwise the same image at
    every chunk depth: a block's k-th hit always goes to partial k mod 4, however the list is
    chunked, and the hits carried across a refill keep their order."""
    require_cuda()
    import numpy as np
    from structsplat_b200.synthetic import make_stress_field
    H = W = 192
    angle = np.random.default_rng(3).uniform(0, np.pi, (H, W)).astype(np.float32)
    f = make_stress_field(H, W, 9000, seed=4, along_edge_angle=angle)
    params = {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}
    images = []
    try:
        for ts in (16, 32):
            for chunk in autotune.CHUNKS:
                _native.call("ss_set_forward_chunk", ts, chunk)
                plan = RenderPlan.for_field(params, H, W, tile_size=ts)
                img = plan.forward(params).clone()
                torch.cuda.synchronize()
                assert not plan.overflowed()
                assert autotune._longest(plan.offsets) > autotune.STAGE_RECORDS
                images.append((ts, img))
    finally:
        for ts in (16, 32):
            _native.call("ss_set_forward_chunk", ts, 0)
    for ts in (16, 32):
        same = [img for t, img in images if t == ts]
        assert all(torch.equal(same[0], img) for img in same[1:]), ts


def test_tuner_picks_a_forward_chunk_for_streamed_lists():
    require_cuda()
    import numpy as np
    from structsplat_b200.synthetic import make_stress_field
    H = W = 192
    angle = np.random.default_rng(3).uniform(0, np.pi, (H, W)).astype(np.float32)
    f = make_stress_field(H, W, 9000, seed=4, along_edge_angle=angle)
    params = {k: torch.tensor(getattr(f, k), device="cuda") for k in PARAM_NAMES}
    go = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    try:
        r = autotune.tune_render(params, H, W, go, repeats=2, use_cache=False)
        assert r.forward_chunk in autotune.CHUNKS
        assert _native.lib().ss_get_forward_chunk(r.tile_size) == r.forward_chunk
        assert any("/chunk" in k for k in r.times_ms)
    finally:
        for ts in (16, 32):
            _native.call("ss_set_forward_chunk", ts, 0)
            _native.call("ss_set_backward_warps", ts, 0)
