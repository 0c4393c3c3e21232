"""Benchmark: forward + backward of the tiled 2D Gaussian rasterizer, ms per iteration.

Workload (default): 1024x1024x3 float32 target from the seeded generator (gratings, polygons,
noise) and 100,000 Gaussians (means uniform, σ = exp(N(ln 2, 0.5)), θ ~ U[0, π), RGB ~ U[0,1]³,
opacity = sigmoid(N(0,1)), 3σ support), normalized mode.  One step = render from the RS field
tensors + gradients of Σ image·(target − 0.5) w.r.t. means, log-scales, rotations, colours and
opacity logits (the reference's fwd+bwd protocol, benchmarks/tiled_render_profile.py:349-351).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Every rank renders its own image (replicas: the path needs no collective); rank 0 prints one
JSON line.  L2 is flushed (a 256 MiB write) before every timed step.  Step times are CUDA-event
durations on the rendering stream, summed over the K steps, max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np
import torch

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

METRIC = "fwd+bwd ms/iter (1024², 100k Gaussians); batched fit img/s vs plain kernel"
WORKLOAD = {"H": 1024, "W": 1024, "N": 100_000, "seed": 0, "mode": "normalized"}
PAIR_SLOTS_FWD, PAIR_SLOTS_BWD = 14, 40   # FP32 issue slots per in-rectangle pair (reference)
BACKWARD_DRAM_BYTES = 40_252_928 + 768  # one backward_kernel launch at this workload (ncu)
# one fused forward + backward tile pass launch at this workload (ncu; bench.py --fused 1)
FUSED_DRAM_BYTES = 23_515_648 + 512
SM_COUNT, FP32_LANES = 148, 128


def measured_peaks():
    try:
        return json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def make_inputs(dev, wl=WORKLOAD):
    from structsplat_b200.synthetic import make_field, make_target
    f = make_field(wl["H"], wl["W"], wl["N"], seed=wl["seed"])
    target = make_target(wl["H"], wl["W"], seed=wl["seed"] + 1)
    host = {"means": f.means, "log_scales": f.log_scales, "rotations": f.rotations,
            "colors": f.colors, "opacity_logits": f.opacity_logits,
            "grad_out": (target - 0.5).astype(np.float32)}
    return host


def pair_count(host, wl=WORKLOAD, dev=None):
    """P = sum over Gaussians of the pixels in their clipped support rectangle (the work unit of
    the roofline): radii from the library's RS projection, rectangles as render.py:62-78 clips
    them (centre rounded half to even, int64)."""
    from structsplat_b200.field import project
    dev = dev or torch.device("cuda")
    t = {k: torch.as_tensor(host[k]).to(dev) for k in ("means", "log_scales", "rotations")}
    n = t["means"].shape[0]
    _, _, radii = project(t["means"], t["log_scales"], t["rotations"],
                          torch.zeros(n, 3, device=dev), None, wl["H"], wl["W"],
                          want_conics=True)
    m = t["means"].double()
    ok = torch.isfinite(m).all(dim=1)
    c = torch.round(torch.where(ok[:, None], m, torch.zeros_like(m))).long()
    lo = torch.clamp(c - radii, min=0)
    hi = torch.minimum(c + radii, torch.tensor([wl["W"] - 1, wl["H"] - 1], device=dev))
    side = torch.clamp(hi - lo + 1, min=0)
    return int((side[:, 0] * side[:, 1] * ok).sum())


def flush_l2(buf):
    buf.fill_(1)   # 256 MiB write, twice the L2


def timed_loop(fn, steps, flush):
    """Per-step CUDA-event times of ``fn`` with an L2 flush before each step."""
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    for i in range(steps):
        flush_l2(flush)
        starts[i].record()
        fn()
        ends[i].record()
    torch.cuda.synchronize()
    return [s.elapsed_time(e) for s, e in zip(starts, ends)]


def run_ours(args, rank, world, dev):
    from structsplat_b200 import _native, render_gaussians
    from structsplat_b200 import render as R
    from structsplat_b200.fit import CapturedStep, RenderPlan

    wl = WORKLOAD
    H, W = wl["H"], wl["W"]
    host = make_inputs(dev)
    names = ["means", "log_scales", "rotations", "colors", "opacity_logits"]
    params = {k: torch.tensor(host[k], device=dev) for k in names}
    grad_out = torch.tensor(host["grad_out"], device=dev)
    normalize = wl["mode"] == "normalized"
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)

    # ---- the measured step: forward + backward as one captured CUDA graph ----
    plan = RenderPlan.for_field(params, H, W, normalize=normalize, fused=args.fused == 1)
    _native.CALLS.clear()
    plan.forward_backward(params, grad_out)
    torch.cuda.synchronize()
    launches_per_step = launches_from_calls(_native.CALLS)
    step = CapturedStep(lambda: plan.forward_backward(params, grad_out), warmup=args.warmup)
    if args.profile:
        for _ in range(args.steps):
            step.replay()
        torch.cuda.synchronize()
        return None
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clocks:
        step_ms = timed_loop(step.replay, args.steps, flush)
    if world > 1:
        torch.distributed.barrier()
    total_ms = sum(step_ms)
    if plan.overflowed():
        raise RuntimeError("tile index capacity exceeded during the timed steps")

    # ---- the additive mode's step (the same field, no normalisation) ----
    plan_add = RenderPlan.for_field(params, H, W, normalize=False, fused=args.fused == 1)
    step_add = CapturedStep(lambda: plan_add.forward_backward(params, grad_out),
                            warmup=args.warmup)
    additive_ms = timed_loop(step_add.replay, args.steps, flush)
    if plan_add.overflowed():
        raise RuntimeError("tile index capacity exceeded during the additive steps")
    del step_add, plan_add

    # ---- the same step through the eager autograd API (render_gaussians + autograd.grad) ----
    leaves = [params[k].clone().requires_grad_(True) for k in names]

    def eager():
        img = render_gaussians(leaves[0], leaves[1], leaves[2], leaves[3], H, W,
                               opacity_logits=leaves[4], normalize=normalize)
        return torch.autograd.grad(img, leaves, grad_out)

    for _ in range(args.warmup):
        eager()
    eager_ms = timed_loop(eager, args.steps, flush)

    # ---- render_field(mode="b200") on precomputed conics / radii / opacities: the call the
    # reference's fit loop makes (fit.py:1043-1056), against its render_cuda_exact arms ----
    from structsplat_b200 import render_field
    from structsplat_b200.field import project
    n = params["means"].shape[0]
    _, conics0, radii0 = project(params["means"], params["log_scales"], params["rotations"],
                                 params["colors"], params["opacity_logits"], H, W,
                                 want_conics=True)
    rf_leaves = [params["means"].clone().requires_grad_(True), conics0.requires_grad_(True),
                 params["colors"].clone().requires_grad_(True),
                 torch.sigmoid(params["opacity_logits"]).requires_grad_(True)]

    def eager_rf():
        img = render_field(rf_leaves[0], rf_leaves[1], rf_leaves[2], radii0, H, W,
                           mode="b200" if normalize else "b200_additive",
                           opacities=rf_leaves[3])
        return torch.autograd.grad(img, rf_leaves, grad_out)

    for _ in range(args.warmup):
        eager_rf()
    eager_rf_ms = timed_loop(eager_rf, args.steps, flush)
    del rf_leaves, conics0, radii0, n

    # ---- dominant kernels alone, CUDA events on the launching stream ----
    kt = {}
    for name, fn in (("forward", plan.render), ("backward_kernel", lambda: plan.backward_tiles(grad_out)),
                     ("backward", lambda: plan.backward(grad_out, params)),
                     ("fused_tile_pass", lambda: plan.tile_pass(grad_out)),
                     ("binning", lambda: (plan.count(), plan.fill())),
                     ("project", lambda: plan.project(params))):
        for _ in range(3):
            fn()
        kt[name] = statistics.median(timed_loop(fn, max(5, args.steps), flush))
    plan.forward(params)
    torch.cuda.synchronize()
    entries = int(plan.offsets[-1].item())

    # ---- end to end with host buffers: H2D inputs, the captured step, D2H gradients ----
    pinned = {k: torch.tensor(host[k]).pin_memory() for k in names + ["grad_out"]}
    grads = plan.grads()
    host_grads = {k: torch.empty(grads[k].shape, dtype=torch.float32).pin_memory() for k in names}
    bi = sum(v.numel() * 4 for v in pinned.values())
    bo = sum(g.numel() * 4 for g in host_grads.values())

    # The step as two graphs, so the 12.6 MB grad_out copy (needed only by the backward) runs
    # on a side stream under the projection, binning and forward; the backward waits for it.
    # Two input slots (device copies of the field and grad_out, each with its own graphs) let
    # step i+1's host-to-device copies run while step i computes and its gradients go back on
    # a third stream: every step still copies its own inputs in and its gradients out.
    slots = [(params, grad_out)] + [({k: params[k].clone() for k in names}, grad_out.clone())]

    def fwd_part(p):
        plan.forward(p, clear_moments=True)

    graphs = [(CapturedStep(lambda p=p: fwd_part(p), warmup=args.warmup),
               CapturedStep(lambda p=p, g=g: plan.backward(g, p, moments_zeroed=True), warmup=1))
              for p, g in slots]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    p_in = [torch.cuda.Event() for _ in slots]
    g_in = [torch.cuda.Event() for _ in slots]
    read_done = [torch.cuda.Event() for _ in slots]
    out_done = [torch.cuda.Event() for _ in slots]

    def e2e_run(k_steps, pipelined):
        main = torch.cuda.current_stream()
        for i in range(k_steps):
            b = i & 1 if pipelined else 0
            p, g = slots[b]
            fwd, bwd = graphs[b]
            # inputs of slot b once the step that last used them has finished reading them
            if i >= (2 if pipelined else 1):
                h2d.wait_event(read_done[b])
            with torch.cuda.stream(h2d):
                for k in names:
                    p[k].copy_(pinned[k], non_blocking=True)
                p_in[b].record(h2d)
                g.copy_(pinned["grad_out"], non_blocking=True)
                g_in[b].record(h2d)
            flush_l2(flush)
            main.wait_event(p_in[b])
            fwd.replay()
            main.wait_event(g_in[b])
            if i:  # the previous step's gradients are on their way out before these overwrite them
                main.wait_event(out_done[(i - 1) & 1 if pipelined else 0])
            bwd.replay()
            read_done[b].record(main)
            with torch.cuda.stream(d2h):
                d2h.wait_event(read_done[b])
                for k in names:
                    host_grads[k].copy_(grads[k], non_blocking=True)
                out_done[b].record(d2h)
        main.wait_stream(h2d)
        main.wait_stream(d2h)

    def e2e_time(pipelined):
        e2e_run(args.warmup, pipelined)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        e2e_run(args.steps, pipelined)
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)

    e2e_serial_total = e2e_time(False)
    e2e_total = e2e_time(True)

    # the copies alone (the same bytes, the same streams, nothing else running): the host link's
    # share of the end-to-end step
    def copies_ms(direction, reps=10):
        times = []
        stream = h2d if direction == "h2d" else d2h
        for _ in range(reps):
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            with torch.cuda.stream(stream):
                if direction == "h2d":
                    for k in names:
                        slots[0][0][k].copy_(pinned[k], non_blocking=True)
                    slots[0][1].copy_(pinned["grad_out"], non_blocking=True)
                else:
                    for k in names:
                        host_grads[k].copy_(grads[k], non_blocking=True)
            t1.record(stream)
            torch.cuda.synchronize()
            times.append(t0.elapsed_time(t1))
        return statistics.median(times)
    h2d_ms, d2h_ms = copies_ms("h2d"), copies_ms("d2h")
    # the split, overlapped steps give the gradients of the one-graph step
    step.replay()
    torch.cuda.synchronize()
    for k in names:
        ref = grads[k].float()
        err = float((host_grads[k].to(dev) - ref).abs().max() / ref.abs().max().clamp_min(1e-30))
        if err > 1e-4:
            raise RuntimeError(f"e2e step gradient {k} differs from the captured step ({err:.2e})")
    del graphs

    step.replay()
    torch.cuda.synchronize()
    step_out = {"image": plan.image.clone(), "grads": {k: v.clone() for k, v in grads.items()}}
    stats = torch.tensor([total_ms, e2e_total, e2e_serial_total, h2d_ms, d2h_ms],
                         dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(stats, op=torch.distributed.ReduceOp.MAX)
    return {"total_ms": float(stats[0]), "e2e_total_ms": float(stats[1]),
            "e2e_serial_total_ms": float(stats[2]), "h2d_ms": float(stats[3]),
            "d2h_ms": float(stats[4]), "step_ms": step_ms,
            "fused": plan.use_fused(), "additive_ms": statistics.median(additive_ms),
            "eager_ms": statistics.median(eager_ms),
            "eager_rf_ms": statistics.median(eager_rf_ms), "kernels_ms": kt, "entries": entries,
            "launches": launches_per_step * args.steps, "bi": bi, "bo": bo,
            "clocks": clocks.summary(), "host": host, "step_out": step_out}


KERNELS_PER_CALL = {
    # kernels of this library launched by each entry point at 1,024 tiles (the index count's
    # last CTA scans the counts up to 4,095 tiles; beyond, a scan kernel follows)
    "ss_project_rs": 1, "ss_pack_splats": 1, "ss_tile_index_count": 1, "ss_tile_index_fill": 3,
    "ss_render_forward": 1, "ss_render_backward": 2, "ss_project_rs_backward": 1,
    "ss_render_backward_moments": 1, "ss_render_backward_finalize_rs": 1,
    "ss_render_forward_backward": 1,
}


def launches_from_calls(calls):
    return sum(KERNELS_PER_CALL.get(k, 1) * v for k, v in calls.items())


def cpu_reference_step_fn(host, wl=WORKLOAD):
    """One fwd+bwd of the reference's CPU (torch) path; the reference package itself when it
    is installed under baseline/_ref, else the oracle's restatement of it."""
    H, W = wl["H"], wl["W"]
    ref_root = REPO / "baseline" / "_ref"
    kind = "port"
    if (ref_root / "structsplat" / "render.py").is_file():
        sys.path.insert(0, str(ref_root))
        from structsplat.gaussians import GaussianField
        from structsplat.render import render_field
        kind = "reference"

        def step():
            f = GaussianField(*[torch.tensor(host[k]) for k in
                                ("means", "log_scales", "rotations", "colors", "opacity_logits")])
            f.trainable()
            img = render_field(f.means, f.conics(), f.colors, f.radii(3.0), H, W,
                               mode=wl["mode"], opacities=f.opacity_values())
            params = [f.means, f.log_scales, f.rotations, f.colors, f.opacities]
            torch.autograd.grad(img, params, torch.tensor(host["grad_out"]))
    else:
        from oracle import field_ref, render_ref

        def step():
            p = [torch.tensor(host[k]).requires_grad_(True) for k in
                 ("means", "log_scales", "rotations", "colors", "opacity_logits")]
            img = render_ref.render(p[0], field_ref.conics(p[1], p[2]), p[3],
                                    field_ref.radii(p[1], p[2], 3.0), H, W,
                                    opacities=torch.sigmoid(p[4]),
                                    normalize=wl["mode"] == "normalized")
            torch.autograd.grad(img, p, torch.tensor(host["grad_out"]))
    return step, kind


def cpu_baseline(host, budget_s=20.0):
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    step, kind = cpu_reference_step_fn(host)
    t0 = time.perf_counter()
    step()
    times = [time.perf_counter() - t0]
    while sum(times) < budget_s * 0.5 and len(times) < 10:
        t0 = time.perf_counter()
        step()
        times.append(time.perf_counter() - t0)
    ms = statistics.median(times[1:] if len(times) > 1 else times) * 1e3
    return {"value": round(ms, 3), "unit": "ms/iter", "cores": threads, "kind": kind,
            "sample": f"{len(times)} full fwd+bwd steps of the same workload (first untimed "
                      "for the median), torch CPU, all host threads"}


def ref_cuda_baseline(host, dev, steps=10, normalize=True):
    """The reference's own CUDA extension (built unmodified for sm_100a into baseline/_ref)
    through its public render_cuda_exact, untiled and tiled arms; None when not built."""
    try:
        sys.path.insert(0, str(REPO / "baseline"))
        from build_ref_cuda import load_reference_extension
        cuda_render = load_reference_extension()
        from structsplat.gaussians import GaussianField
    except Exception as exc:  # not built / not installed
        return {"unavailable": str(exc)[:200]}
    H, W = WORKLOAD["H"], WORKLOAD["W"]
    f = GaussianField(*[torch.tensor(host[k], device=dev) for k in
                        ("means", "log_scales", "rotations", "colors", "opacity_logits")])
    f.trainable()
    params = [f.means, f.log_scales, f.rotations, f.colors, f.opacities]
    go = torch.tensor(host["grad_out"], device=dev)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    res = {}
    for arm, kw in (("cuda", dict(tiled=False)), ("cuda_tiled", dict(tiled=True))):
        def step():
            img = cuda_render.render_cuda_exact(f.means, f.conics(), f.colors, f.radii(3.0), H, W,
                                                opacities=f.opacity_values(),
                                                normalize=normalize, **kw)
            torch.autograd.grad(img, params, go)
        for _ in range(3):
            step()
        times = []
        for _ in range(steps):
            flush_l2(flush)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            step()
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        res[arm] = round(statistics.median(times), 4)
    return res


def _rel(a, b) -> float:
    a = torch.as_tensor(a).detach().double().cpu()
    b = torch.as_tensor(b).detach().double().cpu()
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


def parity_object(host, dev, image, grads, normalize=True):
    """Errors of the timed step's image and RS-field gradients against the reference on the same
    field: its CUDA extension's float32 result (tiled arm, through its own GaussianField and
    render_cuda_exact) and its own renderer evaluated in float64 on the CPU
    (GaussianField.from_numpy(dtype=float64) semantics, render.py:180-235), as max |d| / max |ref|.
    """
    names = ("means", "log_scales", "rotations", "colors", "opacity_logits")
    H, W = WORKLOAD["H"], WORKLOAD["W"]
    out = {"metric": "max |ours - ref| / max |ref| over the image and each gradient"}
    ref_root = REPO / "baseline" / "_ref"
    if not (ref_root / "structsplat" / "render.py").is_file():
        return {"unavailable": "the reference package is not installed under baseline/_ref"}
    if str(ref_root) not in sys.path:
        sys.path.insert(0, str(ref_root))
    from structsplat.gaussians import GaussianField
    from structsplat.render import render_field

    def reference(device, dtype, cuda_ext):
        f = GaussianField(*[torch.tensor(host[k], dtype=dtype, device=device) for k in names])
        f.trainable()
        params = [f.means, f.log_scales, f.rotations, f.colors, f.opacities]
        go = torch.tensor(host["grad_out"], dtype=dtype, device=device)
        if cuda_ext is not None:
            img = cuda_ext.render_cuda_exact(f.means, f.conics(), f.colors, f.radii(3.0), H, W,
                                             opacities=f.opacity_values(), normalize=normalize,
                                             tiled=True)
        else:
            img = render_field(f.means, f.conics(), f.colors, f.radii(3.0), H, W,
                               mode="normalized" if normalize else "additive",
                               opacities=f.opacity_values())
        g = torch.autograd.grad(img, params, go)
        return img.detach(), dict(zip(names, g))

    torch.set_num_threads(os.cpu_count() or 1)
    img64, g64 = reference("cpu", torch.float64, None)
    ours = {"image": image, **grads}
    ref64 = {"image": img64, **g64}
    out["vs_reference_float64"] = {k: round(_rel(ours[k], ref64[k]), 9) for k in ours}
    try:
        sys.path.insert(0, str(REPO / "baseline"))
        from build_ref_cuda import load_reference_extension
        ext = load_reference_extension()
    except Exception as exc:
        out["vs_reference_cuda_float32"] = {"unavailable": str(exc)[:200]}
        return out
    img32, g32 = reference(dev, torch.float32, ext)
    ref32 = {"image": img32, **g32}
    out["vs_reference_cuda_float32"] = {k: round(_rel(ours[k], ref32[k]), 9) for k in ours}
    out["reference_cuda_float32_vs_float64"] = {k: round(_rel(ref32[k], ref64[k]), 9)
                                                for k in ours}
    out["bars"] = {"image": 1e-5, "gradients": 1e-4}
    return out


BATCH_SIZES = [(256, 256), (512, 512), (512, 768), (1024, 1024), (1536, 2048)]  # (H, W)
BATCH_IMAGES, BATCH_DENSITY, BATCH_SEED = 64, 0.1, 7


def _batch_target(args):
    from structsplat_b200.synthetic import make_target
    H, W, seed = args
    return make_target(H, W, seed=seed)


def batched_workload(images=BATCH_IMAGES, seed=BATCH_SEED, rank=0, world=1):
    """The batched-fit workload: image sizes drawn uniformly from BATCH_SIZES, 0.1 Gaussians per
    pixel, seeded targets and fields (targets built in a spawn pool: no fork after CUDA init).
    With several ranks each builds only its share of the images (``shard_images``)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    from structsplat_b200.replicas import shard_images
    from structsplat_b200.synthetic import make_field
    rng = np.random.default_rng(seed)
    all_sizes = [BATCH_SIZES[int(k)] for k in rng.integers(0, len(BATCH_SIZES), images)]
    mine = shard_images(all_sizes, rank, world)
    sizes = [all_sizes[b] for b in mine]
    counts = [int(round(BATCH_DENSITY * h * w)) for h, w in sizes]
    jobs = [(h, w, seed * 1000 + 2 * b) for b, (h, w) in zip(mine, sizes)]
    # the ranks of a node build their shares at the same time: each takes its share of the cores
    workers = max(1, min(16, (os.cpu_count() or 1) // max(world, 1)))
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
        targets = list(pool.map(_batch_target, jobs))
    fields = [make_field(h, w, n, seed=seed * 1000 + 2 * b + 1)
              for b, (h, w), n in zip(mine, sizes, counts)]
    return sizes, counts, targets, fields


def run_batched(args, dev, workload):
    """C4: one batched graph-captured fit step for all images vs looping the per-image step."""
    from structsplat_b200 import _native
    from structsplat_b200.batch import Batch, FitPlan, FitSettings, GraphStep, psnr_from_mse
    names = ["means", "log_scales", "rotations", "colors", "opacity_logits"]
    sizes, counts, targets_np, fields_np = workload
    B = len(sizes)
    targets = [torch.tensor(t, device=dev) for t in targets_np]

    def fresh():
        return [{k: torch.tensor(getattr(f, k), device=dev) for k in names} for f in fields_np]

    settings = FitSettings(fused=_fused_flag(args))
    K, Wm = args.batch_steps, args.warmup

    def timed(fn, iters):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record()
        for _ in range(iters):
            fn()
        e.record()
        torch.cuda.synchronize()
        return s.elapsed_time(e)

    # the launch shape (tile size, backward warps) by the autotuner, timed on this workload; the
    # batched plan and the per-image loops below all use it
    tuned = None
    if not args.no_tune:
        from structsplat_b200 import autotune
        fp = fresh()
        tuned = autotune.tune_fit(sizes, counts, Batch.concat_fields(fp),
                                  Batch(sizes, counts, device=dev).concat_images(targets),
                                  settings, use_cache=False)
        del fp
    ts = tuned.tile_size if tuned else 32

    # batched: one plan for every image, one graph per step
    batch = Batch(sizes, counts, tile_size=ts, device=dev)
    fb = fresh()
    plan = FitPlan(batch, Batch.concat_fields(fb), batch.concat_images(targets), settings)
    step = GraphStep(plan)
    _native.CALLS.clear()
    for _ in range(Wm):
        step.replay()
    with ClockSampler(dev.index) as clocks:
        t_batch = timed(step.replay, K)
    overflow = plan.overflowed()
    _, loss_b = plan.render()
    psnr_b = [psnr_from_mse(m) for m in loss_b[:, 1].tolist()]
    entries = int(plan.offsets[-1].item())
    mem_gb = torch.cuda.max_memory_allocated(dev) / 1e9
    del step, plan

    # per-image loop of the same step (eager launches), the plain per-image kernel
    fl = fresh()
    plans = []
    for b in range(B):
        bb = Batch([sizes[b]], [counts[b]], tile_size=ts, device=dev)
        plans.append(FitPlan(bb, fl[b], targets[b].reshape(-1, 3), settings))

    def loop_step():
        for p in plans:
            p.step()
    # the fit's work per step grows as its Gaussians grow, so the graph loop below starts from
    # the state the eager loop started from
    start = [p.state() for p in plans]
    for _ in range(Wm):
        loop_step()
    t_loop = timed(loop_step, K)
    psnr_l = []
    for p in plans:
        _, loss = p.render()
        psnr_l.append(psnr_from_mse(float(loss[0, 1])))
    # per-image loop with every image's step captured in its own graph (timing only): the same
    # warm-up and steps from the same start, or its first Kg steps against the eager loop's
    Kg = min(K, 100)
    for p, st in zip(plans, start):
        p.restore(st)
    graphs = [GraphStep(p) for p in plans]
    for _ in range(Wm):
        [g.replay() for g in graphs]
    t_loop_graph = timed(lambda: [g.replay() for g in graphs], Kg)
    if Kg < K:  # the eager loop's first Kg steps, from the same start, for a like comparison
        for p, st in zip(plans, start):
            p.restore(st)
        for _ in range(Wm):
            loop_step()
        t_loop_first = timed(loop_step, Kg)
        t_loop_graph *= t_loop / t_loop_first
    del graphs, plans, start

    # ranks fit disjoint shares of the images: the job is as slow as its slowest rank
    from structsplat_b200.replicas import max_over_ranks, sum_over_ranks
    t_batch, t_loop, t_loop_graph, dpsnr = max_over_ranks(
        [t_batch, t_loop, t_loop_graph,
         float(np.max(np.abs(np.array(psnr_b) - np.array(psnr_l))))], device=dev)
    B_all, px_all, g_all, e_all, psum, psum_loop = sum_over_ranks(
        [B, batch.pixels, batch.n, entries, float(np.sum(psnr_b)), float(np.sum(psnr_l))],
        device=dev)
    B_all = int(B_all)
    res = {
        "workload": f"{B_all} images, sizes uniform over {{256x256, 512x512, 768x512, 1024x1024, "
                    f"2048x1536}} (WxH), 0.1 Gaussians/px, seeded generator targets; "
                    f"normalized, pixel MSE, Adam (reference per-group lrs)",
        "images": B_all, "pixels": int(px_all), "gaussians": int(g_all),
        "fused_tile_pass": settings.use_fused(),
        "tile_entries": int(e_all), "steps": K, "warmup": Wm,
        "scaling": "strong (the images are split across ranks)",
        "batched_img_s": round(B_all * K / (t_batch * 1e-3), 1),
        "batched_ms_per_step": round(t_batch / K, 3),
        "loop_eager_img_s": round(B_all * K / (t_loop * 1e-3), 1),
        "loop_graph_img_s": round(B_all * K / (t_loop_graph * 1e-3), 1),
        "psnr_batched_mean": round(psum / max(B_all, 1), 4),
        "psnr_loop_mean": round(psum_loop / max(B_all, 1), 4),
        "psnr_max_abs_diff_vs_loop": round(dpsnr, 6),
        "psnr_after_steps": Wm + K, "index_overflow": overflow,
        "gpu_launches_per_step": 8, "peak_mem_gb": round(mem_gb, 2), "clocks": clocks.summary(),
    }
    res["speedup_vs_loop_eager"] = round(res["batched_img_s"] / res["loop_eager_img_s"], 3)
    if tuned is not None:
        from structsplat_b200 import autotune
        res["autotune"] = autotune.describe(tuned)
    else:
        res["autotune"] = "off (--no-tune): 32-px tiles, default backward warps"
    res["loop_graph_steps"] = Kg
    res["loop_graph_note"] = ("per-image graphs over the first loop_graph_steps steps from the "
                              "eager loop's start, scaled by the eager loop's full/first-steps "
                              "time ratio")
    # Fast mode sums the moments with float atomics, so two runs of the same fit drift apart by
    # rounding over the steps; the deterministic mode's batched and per-image fits are the same
    # iteration, so their PSNRs agree (checked here over the same K steps, both timed): the
    # comparison at equal PSNR (within 0.01 dB) is this pair.
    Kd = K
    dset = FitSettings(deterministic=True)
    fdet = fresh()
    dplan = FitPlan(batch, Batch.concat_fields(fdet), batch.concat_images(targets), dset)
    dstep = GraphStep(dplan)
    t_det = timed(dstep.replay, Kd)
    _, dloss = dplan.render()
    del dstep, dplan
    fdl = fresh()
    dplans = [FitPlan(Batch([sizes[b]], [counts[b]], tile_size=ts, device=dev), fdl[b],
                      targets[b].reshape(-1, 3), dset) for b in range(B)]
    t_det_loop = timed(lambda: [p.step() for p in dplans], Kd)
    dl = [float(p.render()[1][0, 1]) for p in dplans]
    del dplans
    ddiff = float(np.max(np.abs(np.array([psnr_from_mse(m) for m in dloss[:, 1].tolist()]) -
                                np.array([psnr_from_mse(m) for m in dl]))))
    t_det, t_det_loop, ddiff = max_over_ranks([t_det, t_det_loop, ddiff], device=dev)
    res["deterministic"] = {"steps": Kd, "batched_img_s": round(B_all * Kd / (t_det * 1e-3), 1),
                            "loop_eager_img_s": round(B_all * Kd / (t_det_loop * 1e-3), 1),
                            "psnr_max_abs_diff_vs_loop": round(ddiff, 9),
                            "psnr_within_0_01_db": bool(ddiff <= 0.01)}
    res["deterministic"]["speedup_vs_loop_eager"] = round(
        res["deterministic"]["batched_img_s"] / res["deterministic"]["loop_eager_img_s"], 3)
    # the fit step's work: the in-rectangle pairs of every image (forward + backward slots)
    pairs = sum(pair_count({"means": f.means, "log_scales": f.log_scales,
                            "rotations": f.rotations}, {"H": h, "W": w}, dev=dev)
                for f, (h, w) in zip(fields_np, sizes))
    (pairs,) = sum_over_ranks([float(pairs)], device=dev)
    f_mhz = measured_peaks().get("sm_max_mhz") or 1965.0
    peak_slots = SM_COUNT * FP32_LANES * f_mhz * 1e6
    res["pairs_per_step"] = int(pairs)
    res["step_roofline_frac"] = round(
        pairs * (PAIR_SLOTS_FWD + PAIR_SLOTS_BWD) / peak_slots / (t_batch / K * 1e-3), 4)
    world = torch.distributed.get_world_size() if torch.distributed.is_initialized() else 1
    if not args.no_ref_cuda and world == 1:
        res["reference_loop"] = ref_cuda_fit_loop(sizes, counts, targets, fields_np, dev,
                                                  steps=args.ref_batch_steps)
        if "img_s" in res["reference_loop"]:
            res["speedup_vs_reference_loop"] = round(
                res["batched_img_s"] / res["reference_loop"]["img_s"], 2)
    # the reference FitConfig's default loss: 0.7 L1 + 0.3 (1 - SSIM) (config.py:200, 241)
    ws = FitSettings(pixel_loss="l1", ssim_weight=0.3)
    fs = fresh()
    plan = FitPlan(batch, Batch.concat_fields(fs), batch.concat_images(targets), ws)
    step = GraphStep(plan)
    for _ in range(Wm):
        step.replay()
    Ks = min(K, 200)
    t_ssim = timed(step.replay, Ks)
    (t_ssim,) = max_over_ranks([t_ssim], device=dev)
    del step, plan
    res["ssim_loss"] = {"loss": "0.7 l1 + 0.3 (1 - SSIM), 11-tap window", "steps": Ks,
                        "batched_img_s": round(B_all * Ks / (t_ssim * 1e-3), 1),
                        "batched_ms_per_step": round(t_ssim / Ks, 3)}
    if not args.no_ref_cuda and world == 1:
        ref = ref_cuda_fit_loop(sizes, counts, targets, fields_np, dev,
                                steps=args.ref_batch_steps, ssim_weight=0.3)
        res["ssim_loss"]["reference_loop"] = ref
        if "img_s" in ref:
            res["ssim_loss"]["speedup_vs_reference_loop"] = round(
                res["ssim_loss"]["batched_img_s"] / ref["img_s"], 2)
    return res


def ref_cuda_fit_loop(sizes, counts, targets, fields_np, dev, steps=2, ssim_weight=0.0):
    """The reference's plain fit iteration per image (its CUDA extension, tiled arm, through
    render_cuda_exact; pixel MSE — or, with ssim_weight, (1 - w) L1 + w (1 - SSIM) through its
    metrics.ssim with cached target statistics; torch.optim.Adam over its parameter groups;
    log-scale clamp), looped over the images; img/s over `steps` timed passes after one
    warm-up pass."""
    try:
        sys.path.insert(0, str(REPO / "baseline"))
        from build_ref_cuda import load_reference_extension
        cuda_render = load_reference_extension()
        from structsplat.gaussians import GaussianField
        from structsplat import metrics as ref_metrics
    except Exception as exc:
        return {"unavailable": str(exc)[:200]}
    names = ["means", "log_scales", "rotations", "colors", "opacity_logits"]
    runs = []
    for b, f in enumerate(fields_np):
        vals = [f[k] if isinstance(f, dict) else getattr(f, k) for k in names]
        vals = [None if v is None else torch.as_tensor(v, device=dev).clone() for v in vals]
        g = GaussianField(*vals)
        g.trainable()
        groups = g.parameter_groups(5e-2, 3e-2, 1e-2, 3e-2, 1e-2)
        stats = ref_metrics.SSIMTargetStats(targets[b]) if ssim_weight else None
        runs.append((g, torch.optim.Adam(groups), targets[b], sizes[b], stats))

    def one_pass():
        for g, opt, tgt, (H, W), stats in runs:
            img = cuda_render.render_cuda_exact(g.means, g.conics(), g.colors, g.radii(3.0), H, W,
                                                opacities=g.opacity_values(), tiled=True)
            d = img - tgt
            if ssim_weight:
                sv = ref_metrics.ssim(img, tgt, target_stats=stats)
                loss = (1 - ssim_weight) * d.abs().mean(dim=2).mean() + ssim_weight * (1 - sv)
            else:
                loss = (d * d).mean(dim=2).mean()
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            with torch.no_grad():
                g.log_scales.clamp_(max=math.log(max(H, W)))
                g.log_scales.clamp_(min=math.log(0.35))
    one_pass()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(steps):
        one_pass()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e)
    return {"img_s": round(len(runs) * steps / (ms * 1e-3), 2), "steps": steps,
            "ms_per_pass": round(ms / steps, 2), "arm": "cuda_tiled"}


def _fused_flag(args):
    return None if args.fused < 0 else bool(args.fused)


def run_ssim_profile(dev, H=2048, W=2048, calls=13):
    """The SSIM term alone (ss_fit_ssim, w = 0.3, normalized) on one image: ms per call."""
    from structsplat_b200 import _native
    from structsplat_b200.batch import Batch
    from structsplat_b200.render import _p, _stream
    from structsplat_b200.synthetic import make_target
    t = torch.tensor(make_target(H, W, seed=1), device=dev).reshape(-1, 3).contiguous()
    gen = torch.Generator(device=dev).manual_seed(2)
    img = (t + 0.05 * torch.randn(t.shape, device=dev, generator=gen)).clamp(0, 1).contiguous()
    den = torch.rand(H * W, device=dev, generator=gen) + 0.5
    batch = Batch([(H, W)], [0], device=dev)
    wsb = _native.size_query("ss_ssim_workspace_bytes", H * W)
    ws = torch.empty(wsb // 4, device=dev)
    stats = torch.empty(6 * H * W, device=dev)
    _native.call("ss_ssim_target_stats", batch.ref, _p(t), _p(stats), _p(ws), wsb, _stream())
    pg = torch.zeros(H * W, 4, device=dev)
    ssim = torch.zeros(1, device=dev)

    def call():
        _native.call("ss_fit_ssim", batch.ref, _p(img), _p(den), _p(t), _p(stats), 1, 1e-8, 0.3,
                     _p(pg), _p(ssim), _p(ws), wsb, _stream())
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(calls - 3):
        call()
    e.record()
    torch.cuda.synchronize()
    return {"image": f"{W}x{H}", "ms_per_call": round(s.elapsed_time(e) / (calls - 3), 4)}


def st_fp32_slots_per_pixel(grad_sigma: float, tensor_sigma: float) -> int:
    """FP32 issue slots per pixel of the structure tensor of a luma image with central
    gradients: blur taps are a separately rounded multiply and add each (NumPy's order), radii
    round(3 sigma) as structure_tensor.py:61-65 sizes them."""
    rg = max(1, int(round(3.0 * grad_sigma))) if grad_sigma > 0 else 0
    rt = max(1, int(round(3.0 * tensor_sigma))) if tensor_sigma > 0 else 0
    luma, grads, products, eigen = 3, 4, 6, 50
    return luma + 2 * (2 * rg + 1) * 2 + grads + products + 3 * 2 * (2 * rt + 1) * 2 + eigen


ST_CASES = (  # (name, H, W, tensor sigma): the structure tensors the workloads compute
    ("plain_fit_256", 256, 256, 2.0), ("stress_2048", 2048, 2048, 3.0),
    ("placement_1920x1080", 1080, 1920, 2.0))


def run_structure_tensor(dev, calls=20):
    """J = G_rho * (grad I grad I^T) and its eigen-analysis (structure_tensor.compute) on the
    workloads' targets: ms per call, replayed from a CUDA graph (two shared-memory tile kernels,
    the radix select of the energy's median and 99th percentile, the labels), against the
    compulsory HBM traffic (12 B per pixel in, five float32 maps and a uint8 label out: 33 B per
    pixel); the reference's NumPy computation on the host for the 256x256 and 1920x1080
    targets."""
    from structsplat_b200 import structure_tensor as st
    from structsplat_b200.fit import CapturedStep
    from structsplat_b200.synthetic import make_target
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    f_mhz = measured_peaks().get("sm_max_mhz") or 1965.0
    flush = torch.empty(64 << 20, dtype=torch.float32, device=dev)
    out = {"bytes_per_pixel": 33, "peak_gbs": peak,
           "fp32_work": "separately rounded multiply and add per blur tap (NumPy's order), per "
                        "pixel of a luma image: luma 3, sigma blur 2x(2r+1)x2, central "
                        "gradients 4, products 6, rho blur 3x2x(2r+1)x2, eigen-analysis ~50 "
                        "(square root, division, atan2f); peak 148 SMs x 128 FP32 lanes x "
                        "sm_max_mhz"}
    ref_root = REPO / "baseline" / "_ref"
    ref_st = None
    if (ref_root / "structsplat" / "structure_tensor.py").is_file():
        if str(ref_root) not in sys.path:
            sys.path.insert(0, str(ref_root))
        from structsplat import structure_tensor as ref_st
    for name, H, W, rho in ST_CASES:
        tgt = make_target(H, W, seed=61, n_polygons=60 if W == 1920 else 20)
        img = torch.tensor(tgt, device=dev)
        cfg = st.StructureTensorConfig(grad_sigma=1.0, tensor_sigma=rho)
        # captured once (the call's host-side preparation is not timed: a CUDA graph replays
        # its kernels)
        graph = CapturedStep(lambda: st.compute(img, cfg, sync_stats=False), warmup=3)
        times = []
        for _ in range(calls):
            flush_l2(flush)
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            graph.replay()
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        del graph
        ms = statistics.median(times)
        gbs = 33.0 * H * W / (ms * 1e-3) / 1e9
        slots = st_fp32_slots_per_pixel(1.0, rho)
        fp32_ms = slots * H * W / (SM_COUNT * FP32_LANES * f_mhz * 1e6) * 1e3
        hbm_ms = 33.0 * H * W / (peak * 1e9) * 1e3
        row = {"H": H, "W": W, "grad_sigma": 1.0, "tensor_sigma": rho, "ms": round(ms, 4),
               "achieved_gbs": round(gbs, 1), "hbm_frac": round(gbs / peak, 4),
               "fp32_slots_per_pixel": slots, "fp32_frac": round(fp32_ms / ms, 4),
               "bound": "fp32" if fp32_ms > hbm_ms else "hbm",
               "roofline_frac": round(max(fp32_ms, hbm_ms) / ms, 4)}
        if ref_st is not None and H * W <= 1920 * 1080:
            t0 = time.perf_counter()
            ref_st.compute(tgt, ref_st.StructureTensorConfig(grad_sigma=1.0, tensor_sigma=rho))
            row["reference_numpy_ms"] = round((time.perf_counter() - t0) * 1e3, 1)
        out[name] = row
    return out


def run_stress(args, dev):
    """C3: 2048² target, 1M heavy-tailed Gaussians (30% elongated along the structure tensor),
    the whole deterministic Adam fit iteration captured in one CUDA graph."""
    from structsplat_b200 import structure_tensor as st
    from structsplat_b200.batch import Batch, FitPlan, FitSettings, GraphStep, psnr_from_mse
    from structsplat_b200.synthetic import make_stress_field, make_target
    H = W = 2048
    N = 1_000_000
    names = ["means", "log_scales", "rotations", "colors", "opacity_logits"]
    target_np = make_target(H, W, seed=31)
    target = torch.tensor(target_np, device=dev)
    tensor = st.compute(target, st.StructureTensorConfig(grad_sigma=1.0, tensor_sigma=3.0))
    along = (tensor.across_edge_angle + math.pi / 2.0).cpu().numpy()
    f = make_stress_field(H, W, N, seed=32, along_edge_angle=along)
    params = {k: torch.tensor(getattr(f, k), device=dev) for k in names}
    settings = FitSettings(deterministic=True, fused=_fused_flag(args))
    batch = Batch([(H, W)], [N], device=dev)
    plan = FitPlan(batch, params, target.reshape(-1, 3).contiguous(), settings)
    counts = (plan.offsets[1:] - plan.offsets[:-1]).to(torch.int64)
    entries = int(plan.offsets[-1].item())
    host = {"log_scales": f.log_scales, "rotations": f.rotations, "means": f.means}
    pairs = pair_count(host, {"H": H, "W": W})
    _, loss0 = plan.render()
    step = GraphStep(plan)
    for _ in range(args.warmup):
        step.replay()
    K = args.stress_steps
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clocks:
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(K):
            step.replay()
        e.record()
        torch.cuda.synchronize()
    ms = s.elapsed_time(e) / K
    status = int(plan.status.item())
    _, loss1 = plan.render()
    return {"workload": "2048x2048 target, 1M Gaussians, ln-sigma std 1.2, 30% elongated "
                        "(aspect U[5,50]) along structure-tensor orientation (sigma 1, rho 3); "
                        "deterministic two-pass backward; Adam fit iteration in one CUDA graph",
            "ms_per_step": round(ms, 3), "steps": K, "warmup": args.warmup,
            "fused_tile_pass": settings.use_fused(),
            "pairs": pairs, "gpairs_per_s": round(pairs / (ms * 1e-3) / 1e9, 2),
            "step_roofline_frac": round(pairs * (PAIR_SLOTS_FWD + PAIR_SLOTS_BWD) / (
                SM_COUNT * FP32_LANES * (measured_peaks().get("sm_max_mhz") or 1965.0) * 1e6)
                / (ms * 1e-3), 4),
            "roofline_note": "pairs counts every in-rectangle pair, as the reference evaluates "
                             "them; the forward skips 8x8 blocks and the backward skips tile "
                             "entries where every weight underflows to +0 (the elongated "
                             "Gaussians' rectangles), so the fraction can exceed 1",
            "tile_entries": entries, "tile_list_max": int(counts.max()),
            "tile_list_median": float(counts.float().median()),
            "psnr_start": round(psnr_from_mse(float(loss0[0, 1])), 3),
            "psnr_end": round(psnr_from_mse(float(loss1[0, 1])), 3),
            "steps_done": args.warmup + K, "status": status,
            "peak_mem_gb": round(torch.cuda.max_memory_allocated(dev) / 1e9, 2),
            "clocks": clocks.summary()}


def run_e2e_fit(args, dev):
    """C5: 1920x1080 target (60 polygons); structure tensor -> density -> 2M Gaussians placed by
    the seeded sampler -> Adam fit on MSE; time to PSNR thresholds, graph vs plain launches."""
    from structsplat_b200.batch import Batch, FitPlan, FitSettings, GraphStep, psnr_from_mse
    from structsplat_b200.placement import place_field
    from structsplat_b200.synthetic import make_target
    H, W, N = 1080, 1920, 2_000_000
    target = torch.tensor(make_target(H, W, seed=51, n_polygons=60), device=dev)
    thresholds = [float(t) for t in args.psnr_thresholds.split(",")]
    out = {"workload": "1920x1080 target (60 polygons), 2M Gaussians placed from the structure "
                       "tensor (sigma 1, rho 2; aniso_onedge, density_random), normalized MSE, "
                       "Adam with the reference's per-group learning rates",
           "steps": args.e2e_steps, "check_every": args.e2e_check}
    for form in ("graph", "plain"):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t_place = torch.cuda.Event(enable_timing=True)
        t0.record()
        field, _, _ = place_field(target, N, strategy="aniso_onedge", seed=5)
        t_place.record()
        field["opacity_logits"] = None
        batch = Batch([(H, W)], [N], device=dev)
        plan = FitPlan(batch, field, target.reshape(-1, 3).contiguous(),
                       FitSettings(fused=_fused_flag(args)))
        runner = GraphStep(plan).replay if form == "graph" else plan.step
        torch.cuda.synchronize()
        placement_ms = t0.elapsed_time(t_place)
        reached, trace = {}, []
        start = time.perf_counter()
        for it in range(1, args.e2e_steps + 1):
            runner()
            if it % args.e2e_check == 0 or it == args.e2e_steps:
                psnr = psnr_from_mse(float(plan.loss[0, 1]))  # syncs: the check is the timer
                el = time.perf_counter() - start
                trace.append([it, round(psnr, 3), round(el, 3)])
                for t in thresholds:
                    if psnr >= t and str(t) not in reached:
                        reached[str(t)] = {"iter": it, "seconds": round(el, 3)}
        total = time.perf_counter() - start
        out[form] = {"placement_ms": round(placement_ms, 2), "fit_seconds": round(total, 3),
                     "ms_per_step": round(1e3 * total / args.e2e_steps, 3),
                     "time_to_psnr": reached, "trace": trace,
                     "entries": int(plan.offsets[-1].item())}
        if form == "plain" and not args.no_ref_cuda:
            # the reference's own per-launch iteration on the same placed field
            out["reference_cuda_tiled"] = ref_cuda_fit_loop(
                [(H, W)], [N], [target], [{k: v for k, v in field.items()}], dev,
                steps=args.ref_batch_steps)
        del plan, runner
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity object (the reference's float32 and float64 results)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-fit measurement")
    ap.add_argument("--batch-steps", type=int, default=1000)
    ap.add_argument("--ref-batch-steps", type=int, default=2)
    ap.add_argument("--no-tune", action="store_true",
                    help="batched leg: fixed 32-px tiles instead of the autotuner's shape")
    ap.add_argument("--batched-only", action="store_true")
    ap.add_argument("--stress", action="store_true", help="run only the stress workload")
    ap.add_argument("--stress-steps", type=int, default=500)
    ap.add_argument("--no-stress", action="store_true", help="skip the stress leg")
    ap.add_argument("--no-e2e-fit", action="store_true",
                    help="skip the placement + fit end-to-end leg")
    ap.add_argument("--e2e-fit", action="store_true",
                    help="run only the placement + fit end-to-end workload")
    ap.add_argument("--e2e-steps", type=int, default=2000)
    ap.add_argument("--e2e-check", type=int, default=25)
    ap.add_argument("--psnr-thresholds", default="30,33,35,36,37,38,39")
    ap.add_argument("--ssim-profile", action="store_true",
                    help="only time the SSIM term on one 2048x2048 image (for ncu)")
    ap.add_argument("--structure-tensor", action="store_true",
                    help="only time the structure tensor on its three workloads")
    ap.add_argument("--fused", type=int, default=-1, choices=[-1, 0, 1],
                    help="fit legs: forward, loss and backward in one tile pass (1), two (0), "
                         "or the plan's choice (-1: fused in fast mode); the fwd+bwd step: "
                         "one tile pass only with 1")
    ap.add_argument("--dependent-launch", type=int, default=1, choices=[0, 1],
                    help="programmatic dependent launch of the library's kernels (1: on)")
    ap.add_argument("--forward-chunk", type=int, default=0, choices=[0, 64, 128, 256],
                    help="records per streamed forward chunk (0: the library's default)")
    ap.add_argument("--profile", action="store_true",
                    help="only replay the captured step (for ncu launch lists)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "ours":
        from structsplat_b200 import _native
        _native.call("ss_set_dependent_launch", args.dependent_launch)
        for ts in (16, 32):
            _native.call("ss_set_forward_chunk", ts, args.forward_chunk)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        host = make_inputs(None)
        step, kind = cpu_reference_step_fn(host)
        torch.set_num_threads(os.cpu_count() or 1)
        for _ in range(min(args.warmup, 1)):
            step()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step()
        ms = (time.perf_counter() - t0) * 1e3 / args.steps
        line = {"impl": "reference", "metric": METRIC, "value": round(ms, 3), "unit": "ms/iter",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "1024x1024x3, 100k Gaussians, normalized, fwd+bwd through "
                                       "RS params", "parallelism": "cpu"},
                "cpu_baseline": {"value": round(ms, 3), "unit": "ms/iter",
                                 "cores": torch.get_num_threads(), "kind": kind,
                                 "sample": "full workload steps on the host cores"},
                "e2e": {"value": round(ms, 3), "unit": "ms/iter", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=__import__("datetime").timedelta(
            seconds=120))
    if args.ssim_profile:
        dev = torch.device(f"cuda:{local}")
        torch.cuda.set_device(dev)
        print(json.dumps({"ssim_profile": run_ssim_profile(dev)}))
        return
    if args.structure_tensor:
        dev = torch.device(f"cuda:{local}")
        torch.cuda.set_device(dev)
        print(json.dumps({"structure_tensor": run_structure_tensor(dev)}), flush=True)
        return
    if args.stress or args.e2e_fit:
        dev = torch.device(f"cuda:{local}")
        torch.cuda.set_device(dev)
        key, fn = ("stress", run_stress) if args.stress else ("e2e_fit", run_e2e_fit)
        print(json.dumps({key: fn(args, dev)}), flush=True)
        return
    workload = None
    if (args.batched_only or not args.no_batched) and not args.profile:
        # spawn pool before the first CUDA call; each rank builds its share of the images
        workload = batched_workload(rank=rank, world=world)
    dev = torch.device(f"cuda:{local}")
    torch.cuda.set_device(dev)
    if args.batched_only:
        batched = run_batched(args, dev, workload)
        if rank == 0:
            print(json.dumps({"batched": batched}), flush=True)
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    res = run_ours(args, rank, world, dev)
    if res is None:
        return
    batched = run_batched(args, dev, workload) if workload is not None else None
    host = res.pop("host")
    step_out = res.pop("step_out")
    peaks = measured_peaks()
    P = pair_count(host, dev=dev) if rank == 0 else 0
    line = None
    if rank == 0:
        ms = res["total_ms"] / args.steps
        clk = res["clocks"]
        f_mhz = peaks.get("sm_max_mhz") or 1965.0
        peak_slots = SM_COUNT * FP32_LANES * f_mhz * 1e6 / 1e9   # Gslot/s
        kt = res["kernels_ms"]
        bwd_ach = P * PAIR_SLOTS_BWD / (kt["backward_kernel"] * 1e-3) / 1e9
        fwd_ach = P * PAIR_SLOTS_FWD / (kt["forward"] * 1e-3) / 1e9
        fused_ach = P * (PAIR_SLOTS_FWD + PAIR_SLOTS_BWD) / (kt["fused_tile_pass"] * 1e-3) / 1e9
        if res["fused"]:
            roof = {"kernel": "backward_kernel (fused forward + backward tile pass)",
                    "achieved": fused_ach, "traffic": FUSED_DRAM_BYTES,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                      "fused tile pass launch at this workload",
                    "work": f"{PAIR_SLOTS_FWD}+{PAIR_SLOTS_BWD} FP32 issue slots per "
                            f"in-rectangle pair x {P} pairs per launch"}
        else:
            roof = {"kernel": "backward_kernel", "achieved": bwd_ach,
                    "traffic": BACKWARD_DRAM_BYTES,
                    "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                      "backward_kernel launch at this workload",
                    "work": f"{PAIR_SLOTS_BWD} FP32 issue slots per in-rectangle pair x "
                            f"{P} pairs per launch"}
        t_bound_ms = P * (PAIR_SLOTS_FWD + PAIR_SLOTS_BWD) / (peak_slots * 1e9) * 1e3
        line = {
            "metric": METRIC, "value": round(ms, 4), "unit": "ms/iter", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "1024x1024x3 target, 100k Gaussians, normalized, fwd+bwd "
                                   "through RS params (means, log_scales, rotations, colors, "
                                   "opacity logits)", "H": 1024, "W": 1024, "gaussians": 100000,
                       "pairs": P, "tile_entries": res["entries"],
                       "l2": "flushed before every timed step (256 MiB write)",
                       "parallelism": f"replicas x{world}",
                       "dependent_launch": args.dependent_launch,
                       "step": "one captured CUDA graph: RS projection, tile binning, forward, "
                               "backward, RS chain rule",
                       "fused_tile_pass": res["fused"]},
            "roofline": {"bound": "fp32", "kernel": roof["kernel"],
                         "achieved": round(roof["achieved"], 1), "peak": round(peak_slots, 1),
                         "unit": "Gslot/s", "frac": round(roof["achieved"] / peak_slots, 4),
                         "traffic": roof["traffic"], "traffic_source": roof["traffic_source"],
                         "work": roof["work"],
                         "peak_source": "148 SMs x 128 FP32 lanes x sm_max_mhz of "
                                        "MEASURED_PEAKS.json"},
            "backward_kernel_roofline_frac": round(bwd_ach / peak_slots, 4),
            "kernels_ms": {k: round(v, 4) for k, v in kt.items()},
            "eager_autograd_ms_per_step": round(res["eager_ms"], 4),
            "eager_render_field_ms_per_step": round(res["eager_rf_ms"], 4),
            "forward_roofline_frac": round(fwd_ach / peak_slots, 4),
            "step_roofline_frac": round(t_bound_ms / ms, 4),
            "clocks": clk,
            "gpu_launches": res["launches"],
            "e2e": {"value": round(res["e2e_total_ms"] / args.steps, 4), "unit": "ms/iter",
                    "h2d_bytes_per_step": res["bi"], "d2h_bytes_per_step": res["bo"],
                    "copies": "pinned host buffers; per step the field and grad_out H2D on a "
                              "copy stream into one of two device input slots (step i+1's "
                              "copies run under step i), the forward waits for the field, the "
                              "backward for grad_out; gradients D2H on a third stream",
                    "serial_ms_per_step": round(res["e2e_serial_total_ms"] / args.steps, 4),
                    "h2d_alone_ms": round(res["h2d_ms"], 4),
                    "d2h_alone_ms": round(res["d2h_ms"], 4),
                    "h2d_gbs": round(res["bi"] / (res["h2d_ms"] * 1e-3) / 1e9, 2),
                    "d2h_gbs": round(res["bo"] / (res["d2h_ms"] * 1e-3) / 1e9, 2),
                    # the slowest of the three overlapped legs bounds a step
                    "bound_ms": round(max(res["h2d_ms"], res["d2h_ms"], ms), 4),
                    "frac_of_bound": round(max(res["h2d_ms"], res["d2h_ms"], ms) /
                                           (res["e2e_total_ms"] / args.steps), 4)},
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(host)
        line["additive"] = {"ms_per_step": round(res["additive_ms"], 4),
                            "step": "the same captured step with normalize=False"}
        if world == 1 and not args.no_ref_cuda:
            line["reference_cuda_ms"] = ref_cuda_baseline(host, dev)
            line["additive"]["reference_cuda_ms"] = ref_cuda_baseline(host, dev,
                                                                      normalize=False)
        if batched is not None:
            line["batched"] = batched
        if world == 1 and not args.no_parity:
            line["parity"] = parity_object(host, dev, step_out["image"], step_out["grads"])
        del step_out
        torch.cuda.empty_cache()
        if world == 1:
            line["structure_tensor"] = run_structure_tensor(dev)
        if world == 1 and not args.no_stress:
            line["stress"] = run_stress(args, dev)
            torch.cuda.empty_cache()
        if world == 1 and not args.no_e2e_fit:
            line["e2e_fit"] = run_e2e_fit(args, dev)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
