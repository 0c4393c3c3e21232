"""Autotuner for the render launch shape: tile size and warps per backward tile.

The reference renders with one fixed shape (16x16 tiles, ``cuda_render.py:258``).  Here each
workload picks, by timing on the GPU it runs on, among

* render tile 16 or 32 (pixels per CTA; also the staging depth: a 32x32 tile stages its whole
  list up to 512 Gaussians for the forward and 448 for the backward, a 16x16 tile up to 512,
  longer lists stream through 64-record chunks), and
* warps per backward CTA (4 or 8 for tile 16, 8 or 16 for tile 32), and
* when the workload's longest tile list is longer than the forward's 512-record stage (the
  list then streams through two chunks), the forward's chunk depth: 64, 128 or 256 records,
  timed at the chosen shape.

The forward's threads follow the tile (one warp per 8x8 block).  Timing runs the render forward
and backward of the actual workload (the field and images in hand), median of a few CUDA-event
timed repeats per candidate.  Results are cached per workload signature and device in a JSON
file (``$STRUCTSPLAT_B200_TUNE_CACHE``, default ``~/.cache/structsplat_b200/tune.json``).
Which shape is chosen never changes an image; in deterministic mode the gradient's summation
order follows the tile size, so deterministic results are reproducible for a fixed shape.
"""
from __future__ import annotations

import json
import math
import os
import statistics
from dataclasses import asdict, dataclass, field
from pathlib import Path

import torch

from . import _native

CANDIDATES = ((16, 4), (16, 8), (32, 8), (32, 16))
CHUNKS = (64, 128, 256)  # forward records per streamed chunk
STAGE_RECORDS = 512      # the forward's whole-list stage


@dataclass
class TuneResult:
    tile_size: int
    backward_warps: int
    key: str
    times_ms: dict = field(default_factory=dict)
    cached: bool = False
    forward_chunk: int = 0  # 0: the library's default (lists short enough not to stream)

    def apply(self):
        """Make this shape the one the library launches (the knobs are process-wide)."""
        _native.call("ss_set_backward_warps", self.tile_size, self.backward_warps)
        _native.call("ss_set_forward_chunk", self.tile_size, self.forward_chunk)
        return self


def cache_path() -> Path:
    env = os.environ.get("STRUCTSPLAT_B200_TUNE_CACHE")
    return Path(env) if env else Path.home() / ".cache" / "structsplat_b200" / "tune.json"


def _load():
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store(key, result: TuneResult):
    data = _load()
    data[key] = {"tile_size": result.tile_size, "backward_warps": result.backward_warps,
                 "forward_chunk": result.forward_chunk, "times_ms": result.times_ms}
    try:
        p = cache_path()
        p.parent.mkdir(parents=True, exist_ok=True)
        tmp = p.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(p)
    except OSError:
        pass  # a read-only home only costs a re-tune


def _bucket(x: float) -> str:
    """Two significant digits on a log scale: workloads within ~10% share a key."""
    if x <= 0:
        return "0"
    return f"{10 ** (round(math.log10(x) * 20) / 20):.3g}"


def workload_key(pixels: int, gaussians: int, entries: int, images: int, normalize: bool,
                 fade: bool, deterministic: bool, fit: bool, fused: bool = False) -> str:
    dev = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    parts = [dev, f"px={_bucket(pixels)}", f"g/px={_bucket(gaussians / max(pixels, 1))}",
             f"e/g={_bucket(entries / max(gaussians, 1))}", f"img={_bucket(images)}",
             f"norm={int(normalize)}", f"fade={int(fade)}", f"det={int(deterministic)}",
             f"fit={int(fit)}"]
    if fused:
        parts.append("fused=1")
    return "|".join(parts)


def _time(fn, repeats: int) -> float:
    fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(repeats):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        torch.cuda.synchronize()
        times.append(s.elapsed_time(e))
    return statistics.median(times)


def _pick(key, candidates, build, repeats, use_cache, longest=None) -> TuneResult:
    """The fastest (tile, warps) candidate; then, when ``longest(ts)`` (the longest tile list
    at that tile size) exceeds the forward's stage, the fastest forward chunk at that shape."""
    if use_cache:
        hit = _load().get(key)
        if hit and (hit["tile_size"], hit["backward_warps"]) in set(candidates):
            return TuneResult(hit["tile_size"], hit["backward_warps"], key, hit["times_ms"],
                              cached=True, forward_chunk=hit.get("forward_chunk", 0)).apply()
    before = {ts: (_native.lib().ss_get_backward_warps(ts),
                   _native.lib().ss_get_forward_chunk(ts)) for ts in (16, 32)}
    times = {}
    chunk = 0
    try:
        for ts, warps in candidates:
            _native.call("ss_set_backward_warps", ts, warps)
            times[f"{ts}x{warps}"] = round(_time(build(ts), repeats), 4)
        best = min(times, key=times.get)
        ts, warps = (int(v) for v in best.split("x"))
        if longest is not None and longest(ts) > STAGE_RECORDS:
            _native.call("ss_set_backward_warps", ts, warps)
            chunk_times = {}
            for c in CHUNKS:
                _native.call("ss_set_forward_chunk", ts, c)
                chunk_times[c] = round(_time(build(ts), repeats), 4)
                times[f"{ts}x{warps}/chunk{c}"] = chunk_times[c]
            chunk = min(chunk_times, key=chunk_times.get)
    finally:
        for t, (w, c) in before.items():
            _native.call("ss_set_backward_warps", t, w)
            _native.call("ss_set_forward_chunk", t, c)
    result = TuneResult(ts, warps, key, times, forward_chunk=chunk).apply()
    if use_cache:
        _store(key, result)
    return result


def _longest(offsets: torch.Tensor) -> int:
    return int((offsets[1:] - offsets[:-1]).max().item()) if offsets.numel() > 1 else 0


def tune_render(params: dict, H: int, W: int, grad_out: torch.Tensor, normalize: bool = True,
                deterministic: bool = False, candidates=CANDIDATES, repeats: int = 5,
                use_cache: bool = True) -> TuneResult:
    """Best shape for one image's render forward + backward (``fit.RenderPlan``)."""
    from .fit import RenderPlan
    plans = {}

    def build(ts):
        if ts not in plans:
            plans[ts] = RenderPlan.for_field(params, H, W, normalize=normalize,
                                             deterministic=deterministic, tile_size=ts)
        plan = plans[ts]
        plan.forward(params)
        return lambda: (plan.render(), plan.backward(grad_out, params))

    build(candidates[0][0])
    entries = int(plans[candidates[0][0]].offsets[-1].item())
    key = workload_key(H * W, params["means"].shape[0], entries, 1, normalize, False,
                       deterministic, fit=False)
    return _pick(key, candidates, build, repeats, use_cache,
                 longest=lambda ts: _longest(plans[ts].offsets))


def tune_fit(sizes, counts, params: dict, target: torch.Tensor, settings=None,
             candidates=CANDIDATES, repeats: int = 5, use_cache: bool = True) -> TuneResult:
    """Best shape for a (batched) fit iteration's forward-with-loss + backward."""
    from .batch import Batch, FitPlan, FitSettings
    settings = settings or FitSettings()
    plans = {}

    def build(ts):
        if ts not in plans:
            batch = Batch(sizes, counts, tile_size=ts, device=target.device)
            plan = FitPlan(batch, params, target, settings)
            plan.project()
            plan.count()
            plan.fill()
            plans[ts] = plan
        plan = plans[ts]

        def run():
            if plan.s.use_fused():
                plan.forward_backward()
            else:
                plan.forward_loss()
                plan.backward()
        return run

    try:
        build(candidates[0][0])
        entries = int(plans[candidates[0][0]].offsets[-1].item())
        pixels = sum(h * w for h, w in sizes)
        key = workload_key(pixels, sum(counts), entries, len(sizes), settings.normalize,
                           settings.fade_alpha > 0, settings.deterministic, fit=True,
                           fused=settings.use_fused())
        # the fused fit pass streams through the backward's stage, which has no chunk knob
        longest = None if settings.use_fused() else (lambda ts: _longest(plans[ts].offsets))
        return _pick(key, candidates, build, repeats, use_cache, longest=longest)
    finally:
        for plan in plans.values():  # the probe backward added into the moments: clear them
            plan.bwd_ws.zero_()


def describe(result: TuneResult) -> dict:
    d = asdict(result)
    d.pop("key")
    return d
