"""Batched, graph-captured Adam fitting of many independent images.

The reference fits one image per ``fit`` call (``fit.py:2697``); its plain iteration is render →
pixel loss (``fit.py:800-814``) → backward → ``torch.optim.Adam`` over the five parameter groups
(``gaussians.py:203-214``, ``fit.py:672-682``) → log-scale clamp (``fit.py:3033, 3359-3366``).

Here B images of any sizes form one ``Batch``: their tiles are numbered as one tile set (image
by image), their Gaussians are concatenated, and every stage of the iteration is ONE launch for
the whole batch — projection, tile count, fill + sort, a forward that also evaluates the loss and
writes the backward's per-pixel input, the backward into per-Gaussian moments, and one fused
update kernel (moments → gradients → RS chain rule → Adam → clamp).  The whole iteration is
captured in a CUDA graph, so a step costs one graph launch however many images there are.
Every image renders exactly as it would alone (same tile lists, same ascending order), so a
batch of one image is the single-image fit.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import torch

from . import _native
from .render import DEFAULT_EPS, RECORD_FLOATS, RENDER_TILE, _p, _stream, fade_tail, validate_eps

PARAM_NAMES = ("means", "log_scales", "rotations", "colors", "opacity_logits")
LOSS_KINDS = {"l1": 0, "l2": 1, "charbonnier": 2}


class Batch:
    """Device tables of a batch of images (``ss_batch`` in the C header)."""

    def __init__(self, sizes, counts, tile_size: int = RENDER_TILE, device="cuda"):
        if len(sizes) != len(counts) or not sizes:
            raise ValueError("a batch needs one (H, W) size and one Gaussian count per image")
        self.sizes = [(int(h), int(w)) for h, w in sizes]
        self.counts = [int(c) for c in counts]
        if any(h < 0 or w < 0 for h, w in self.sizes) or any(c < 0 for c in self.counts):
            raise ValueError("negative image size or Gaussian count")
        self.tile_size = int(tile_size)
        self.device = torch.device(device)
        ts = self.tile_size
        table, pixel_base, tile_image = [], [], []
        first_tile, first_pixel = 0, 0
        for b, (h, w) in enumerate(self.sizes):
            tx, ty = (w + ts - 1) // ts, (h + ts - 1) // ts
            table.append([h, w, tx, first_tile])
            pixel_base.append(first_pixel)
            tile_image.append(torch.full((tx * ty,), b, dtype=torch.int32))
            first_tile += tx * ty
            first_pixel += h * w
        self.tiles, self.pixels = first_tile, first_pixel
        self.n = sum(self.counts)
        gb = [0]
        for c in self.counts:
            gb.append(gb[-1] + c)
        self.gaussian_base_host = gb
        self.pixel_base_host = pixel_base
        d = self.device
        self.image_table = torch.tensor(table, dtype=torch.int32, device=d)
        self.pixel_base = torch.tensor(pixel_base, dtype=torch.int64, device=d)
        self.gaussian_base = torch.tensor(gb, dtype=torch.int32, device=d)
        self.gaussian_image = torch.repeat_interleave(
            torch.arange(len(self.sizes), dtype=torch.int32),
            torch.tensor(self.counts, dtype=torch.int64)).to(d)
        self.tile_image = torch.cat(tile_image).to(d) if self.tiles else torch.zeros(
            1, dtype=torch.int32, device=d)
        self.struct = _native.SsBatch(
            images=len(self.sizes), tile_size=ts, tiles=self.tiles, pixels=self.pixels,
            image_table=self.image_table.data_ptr(), pixel_base=self.pixel_base.data_ptr(),
            gaussian_base=self.gaussian_base.data_ptr(),
            gaussian_image=self.gaussian_image.data_ptr() if self.n else None,
            tile_image=self.tile_image.data_ptr())
        self.ref = ctypes.byref(self.struct)

    @property
    def images(self) -> int:
        return len(self.sizes)

    def pixel_slice(self, b: int) -> slice:
        h, w = self.sizes[b]
        return slice(self.pixel_base_host[b], self.pixel_base_host[b] + h * w)

    def gaussian_slice(self, b: int) -> slice:
        return slice(self.gaussian_base_host[b], self.gaussian_base_host[b + 1])

    def split_images(self, flat: torch.Tensor):
        """(P, C) concatenated rows → list of (H, W, C) views."""
        c = flat.shape[-1] if flat.dim() > 1 else 1
        return [flat[self.pixel_slice(b)].view(h, w, c) for b, (h, w) in enumerate(self.sizes)]

    def concat_images(self, images) -> torch.Tensor:
        return torch.cat([im.reshape(-1, im.shape[-1]) for im in images]).contiguous()

    @staticmethod
    def concat_fields(fields) -> dict:
        out = {}
        for k in PARAM_NAMES:
            parts = [f.get(k) for f in fields]
            if any(p is None for p in parts):
                if not all(p is None for p in parts):
                    raise ValueError(f"{k} must be given for every field or none")
                out[k] = None
            else:
                out[k] = torch.cat(parts).contiguous()
        return out


@dataclass
class FitSettings:
    """The plain fit's knobs (``FitConfig`` defaults, config.py:188-266)."""
    lr_means: float = 5e-2
    lr_scales: float = 3e-2
    lr_rot: float = 1e-2
    lr_color: float = 3e-2
    lr_opacity: float = 1e-2
    pixel_loss: str = "l2"
    charbonnier_eps: float = 1e-3
    # weight w of the SSIM term, loss = (1 - w) pixel_loss + w (1 - SSIM) (fit.py:3244); the
    # reference's FitConfig default is 0.3 with pixel_loss "l1" (config.py:200, 241), its plain
    # method MSE alone (w = 0)
    ssim_weight: float = 0.0
    normalize: bool = True
    eps: float = DEFAULT_EPS
    sigma_cutoff: float = 3.0
    dilation: float = 0.0
    fade_alpha: float = 0.0
    deterministic: bool = False
    # one tile kernel for forward, loss and backward (the same numbers as the two-kernel step);
    # None: fused in fast mode, two kernels in deterministic mode (where the fused kernel's extra
    # registers spill: 9.75 vs 9.65 ms on the 2048^2 / 1 M stress step, 8.79 vs 9.20 ms fused
    # on the 64-image batched step)
    fused: bool | None = None

    def use_fused(self) -> bool:
        return (not self.deterministic) if self.fused is None else bool(self.fused)
    betas: tuple = (0.9, 0.999)
    adam_eps: float = 1e-8
    scale_min: float = 0.35  # log-scale floor ln(0.35) (fit.py:3033)

    @classmethod
    def uniform_lr(cls, lr: float, **kw) -> "FitSettings":
        return cls(lr_means=lr, lr_scales=lr, lr_rot=lr, lr_color=lr, lr_opacity=lr, **kw)

    def lrs(self):
        return [self.lr_means, self.lr_scales, self.lr_rot, self.lr_color, self.lr_opacity]


class FitPlan:
    """Every buffer of a batched fit iteration, allocated once; ``step()`` only launches."""

    def __init__(self, batch: Batch, params: dict, target: torch.Tensor,
                 settings: FitSettings | None = None, capacity: int = 0):
        self.batch = batch
        self.s = s = settings or FitSettings()
        if s.pixel_loss not in LOSS_KINDS:
            raise ValueError(f"unknown pixel_loss {s.pixel_loss!r}; expected l1, l2, or charbonnier")
        if s.normalize:
            validate_eps(s.eps)
        self.params = params
        self.has_opacity = params.get("opacity_logits") is not None
        n, d = batch.n, batch.device
        for k in PARAM_NAMES:
            t = params.get(k)
            if t is not None and (t.device.type != "cuda" or t.dtype != torch.float32
                                  or not t.is_contiguous() or t.shape[0] != n):
                raise ValueError(f"{k} must be a contiguous CUDA float32 tensor with {n} rows")
        if target.shape != (batch.pixels, 3) or not target.is_contiguous():
            raise ValueError("target must be the contiguous (P, 3) concatenation of the images")
        self.target = target
        self.n = n
        self.tail = fade_tail(s.sigma_cutoff, s.fade_alpha)
        self.cull = s.fade_alpha >= 1.0
        f32 = dict(device=d, dtype=torch.float32)
        self.records = torch.empty(max(n, 1) * RECORD_FLOATS, **f32)
        self.offsets = torch.zeros(batch.tiles + 1, device=d, dtype=torch.int32)
        self.status = torch.zeros(1, device=d, dtype=torch.int32)
        self.idx_ws_bytes = _native.size_query("ss_batch_tile_index_workspace_bytes", batch.ref, n)
        self.idx_ws = torch.empty(max(self.idx_ws_bytes, 1), device=d, dtype=torch.uint8)
        if capacity <= 0:
            capacity = self.measure_entries() * 3 // 2 + 4096
        self.capacity = int(capacity)
        self.gids = torch.empty(self.capacity, device=d, dtype=torch.int32)
        self.bwd_ws_bytes = _native.size_query("ss_fit_backward_workspace_bytes", n,
                                               self.capacity, int(s.deterministic))
        self.bwd_ws = torch.zeros(max(self.bwd_ws_bytes // 4, 4), **f32)
        self.pixel_grad = torch.empty(max(batch.pixels, 1), 4, **f32)
        self.loss = torch.zeros(batch.images, 2, **f32)
        if not 0.0 <= s.ssim_weight <= 1.0:
            raise ValueError(f"ssim_weight must lie in [0, 1], got {s.ssim_weight}")
        if s.ssim_weight > 0.0:  # the SSIM term needs the whole image before the backward
            P = max(batch.pixels, 1)
            self.image = torch.empty(P, 3, **f32)
            self.den = torch.empty(P, **f32)
            self.ssim = torch.zeros(batch.images, **f32)
            self.ssim_stats = torch.empty(6 * P, **f32)
            self.ssim_ws_bytes = _native.size_query("ss_ssim_workspace_bytes", batch.pixels)
            self.ssim_ws = torch.empty(max(self.ssim_ws_bytes // 4, 1), **f32)
            _native.call("ss_ssim_target_stats", batch.ref, _p(target), _p(self.ssim_stats),
                         _p(self.ssim_ws), self.ssim_ws_bytes, _stream())
        self.exp_avg = {k: torch.zeros_like(v) for k, v in params.items() if v is not None}
        self.exp_avg_sq = {k: torch.zeros_like(v) for k, v in params.items() if v is not None}
        self.step_state = torch.zeros(2, device=d, dtype=torch.int32)
        self.log_hi = torch.tensor([math.log(max(h, w, 1)) for h, w in batch.sizes], **f32)
        self._ptr_arrays()

    def _ptr_arrays(self):
        def arr(dct):
            a = (ctypes.c_void_p * 5)()
            for i, k in enumerate(PARAM_NAMES):
                t = dct.get(k)
                a[i] = t.data_ptr() if t is not None else None
            return a
        self._p_params = arr(self.params)
        self._p_m = arr(self.exp_avg)
        self._p_v = arr(self.exp_avg_sq)
        self._lrs = (ctypes.c_double * 5)(*self.s.lrs())

    def measure_entries(self) -> int:
        """Tile-list total of the current field (one host sync)."""
        self.project()
        self.count()
        return int(self.offsets[-1].item())

    # -- stages ------------------------------------------------------------------------
    def project(self):
        p = self.params
        _native.call("ss_batch_project_rs", self.batch.ref, _p(p["means"]), _p(p["log_scales"]),
                     _p(p["rotations"]), _p(p["colors"]), _p(p.get("opacity_logits")), self.n,
                     float(self.s.dilation), float(self.s.sigma_cutoff), _p(self.records),
                     _stream())

    def count(self):
        _native.call("ss_batch_tile_index_count", self.batch.ref, _p(self.records), self.n,
                     int(self.cull), float(self.s.sigma_cutoff), _p(self.offsets), _p(self.idx_ws),
                     self.idx_ws_bytes, _p(self.status), _stream())

    def project_count(self):
        """project() and count() in one kernel (ss_batch_project_rs_index_count)."""
        p = self.params
        _native.call("ss_batch_project_rs_index_count", self.batch.ref, _p(p["means"]),
                     _p(p["log_scales"]), _p(p["rotations"]), _p(p["colors"]),
                     _p(p.get("opacity_logits")), self.n, float(self.s.dilation),
                     float(self.s.sigma_cutoff), int(self.cull), _p(self.records),
                     _p(self.offsets), _p(self.idx_ws), self.idx_ws_bytes, None, 0,
                     _p(self.status), _stream())

    def fill(self):
        _native.call("ss_batch_tile_index_fill", self.batch.ref, _p(self.records), self.n,
                     int(self.cull), float(self.s.sigma_cutoff), _p(self.offsets), _p(self.gids),
                     self.capacity, _p(self.idx_ws), self.idx_ws_bytes, _p(self.status),
                     _stream())

    def forward_loss(self, image=None, den=None):
        s = self.s
        _native.call("ss_fit_forward_loss", self.batch.ref, _p(self.records), self.n,
                     _p(self.gids), self.capacity, _p(self.offsets), int(s.normalize),
                     float(s.eps), float(self.tail), _p(self.target), LOSS_KINDS[s.pixel_loss],
                     float(s.charbonnier_eps), _p(self.pixel_grad), _p(image), _p(den),
                     _p(self.loss), _p(self.status), _stream())

    def backward(self):
        _native.call("ss_fit_backward", self.batch.ref, _p(self.records), self.n, _p(self.gids),
                     self.capacity, _p(self.offsets), float(self.tail), _p(self.pixel_grad),
                     int(self.s.deterministic), _p(self.bwd_ws), self.bwd_ws_bytes,
                     _p(self.status), _stream())

    def forward_backward(self):
        """Forward, pixel loss and backward of every tile in one kernel (the loss gradient stays
        on chip); the same images, losses and moments as forward_loss() + backward()."""
        s = self.s
        _native.call("ss_fit_forward_backward", self.batch.ref, _p(self.records), self.n,
                     _p(self.gids), self.capacity, _p(self.offsets), int(s.normalize),
                     float(s.eps), float(self.tail), _p(self.target), LOSS_KINDS[s.pixel_loss],
                     float(s.charbonnier_eps), None, None, _p(self.loss),
                     int(s.deterministic), _p(self.bwd_ws), self.bwd_ws_bytes, _p(self.status),
                     _stream())

    def ssim_term(self):
        """Mixes the SSIM term into pixel_grad after forward_loss wrote the image and den."""
        s = self.s
        _native.call("ss_fit_ssim", self.batch.ref, _p(self.image), _p(self.den),
                     _p(self.target), _p(self.ssim_stats), int(s.normalize), float(s.eps),
                     float(s.ssim_weight), _p(self.pixel_grad), _p(self.ssim), _p(self.ssim_ws),
                     self.ssim_ws_bytes, _stream())

    def update(self):
        s = self.s
        _native.call("ss_fit_adam_update", self.batch.ref, _p(self.records), self.n,
                     _p(self.gids), self.capacity, _p(self.offsets), int(s.deterministic),
                     _p(self.bwd_ws), float(s.dilation), self._p_params, self._p_m, self._p_v,
                     self._lrs, float(s.betas[0]), float(s.betas[1]), float(s.adam_eps),
                     float(math.log(s.scale_min)), _p(self.log_hi), _p(self.step_state),
                     _stream())

    def step(self):
        """One fit iteration for every image of the batch."""
        self.loss.zero_()
        self.project_count()
        self.fill()
        if self.s.ssim_weight > 0.0:
            self.ssim.zero_()
            self.forward_loss(image=self.image, den=self.den)
            self.ssim_term()
            self.backward()
        elif self.s.use_fused():
            self.forward_backward()
        else:
            self.forward_loss()
            self.backward()
        self.update()

    def render(self):
        """Current images (P,3) and the per-image [loss, mse] of the current field."""
        image = torch.empty(max(self.batch.pixels, 1), 3, device=self.target.device)
        self.loss.zero_()
        self.project_count()
        self.fill()
        self.forward_loss(image=image)
        return image[: self.batch.pixels], self.loss.clone()

    def overflowed(self) -> bool:
        return bool(int(self.status.item()) & 1)

    def gradients(self) -> dict:
        """The parameter gradients the last ``update()`` fed to Adam, as views into the fit
        workspace: means (N,2), log_scales (N,2), rotations (N,), colors (N,3) and
        opacity_logits (N,) (None without opacities).  They sit at the end of the workspace in
        five 256-byte-aligned arrays (``fit_grads_layout`` of the CUDA library)."""
        n = self.n

        def a256(x):
            return (x + 255) // 256 * 256
        sizes = [a256(8 * n), a256(8 * n), a256(4 * n), a256(12 * n), a256(4 * n)]
        off = (self.bwd_ws_bytes - sum(sizes)) // 4
        out = {}
        for k, shape, sz in zip(PARAM_NAMES, [(n, 2), (n, 2), (n,), (n, 3), (n,)], sizes):
            count = 1
            for d in shape:
                count *= d
            out[k] = self.bwd_ws[off:off + count].view(shape)
            off += sz // 4
        if not self.has_opacity:
            out["opacity_logits"] = None
        return out

    def state(self):
        """Snapshot of the optimisation state (field, Adam moments, step)."""
        keep = {k: v.clone() for k, v in self.params.items() if v is not None}
        return (keep, {k: v.clone() for k, v in self.exp_avg.items()},
                {k: v.clone() for k, v in self.exp_avg_sq.items()}, self.step_state.clone())

    def restore(self, snap):
        p, m, v, st = snap
        for k, t in p.items():
            self.params[k].copy_(t)
        for k, t in m.items():
            self.exp_avg[k].copy_(t)
        for k, t in v.items():
            self.exp_avg_sq[k].copy_(t)
        self.step_state.copy_(st)


def psnr_from_mse(mse: float) -> float:
    return 10.0 * math.log10(1.0 / max(float(mse), 1e-20))


class GraphStep:
    """A FitPlan step captured in a CUDA graph (warm-up on a side stream first)."""

    def __init__(self, plan: FitPlan):
        snap = plan.state()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            plan.step()
        torch.cuda.current_stream().wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            plan.step()
        plan.restore(snap)
        if not plan.s.deterministic:
            plan.bwd_ws.zero_()
        self.plan = plan

    def replay(self):
        self.graph.replay()


def fit_batch(fields, targets, iters: int = 100, settings: FitSettings | None = None,
              graph: bool = True, log_every: int = 0, check_every: int = 50,
              tile_size: int = RENDER_TILE, tune: bool = False):
    """Fit B independent fields to B targets (H_b, W_b, 3) in one batch.

    ``fields`` is a list of dicts of CUDA float32 tensors (the five ``PARAM_NAMES``; opacity
    logits may be None for all), updated in place.  Returns a history with, per logged
    iteration, every image's PSNR of the pre-update render, the final PSNR per image, and the
    plan.  Every ``check_every`` steps the host reads the index status; if the tile list
    outgrew its capacity the plan is rebuilt with more room (in deterministic mode the steps
    since the last check are replayed from a snapshot, so the result never depends on it).
    ``tune=True`` lets the autotuner pick the tile size and backward warps for this workload
    (``autotune.tune_fit``) instead of ``tile_size``.
    """
    settings = settings or FitSettings()
    sizes = [(int(t.shape[0]), int(t.shape[1])) for t in targets]
    counts = [int(f["means"].shape[0]) for f in fields]
    params = Batch.concat_fields(fields)
    target = torch.cat([t.reshape(-1, 3) for t in targets]).contiguous()
    tuned = None
    if tune:
        from .autotune import tune_fit
        tuned = tune_fit(sizes, counts, params, target, settings)
        tile_size = tuned.tile_size
    batch = Batch(sizes, counts, tile_size=tile_size, device=targets[0].device)
    plan = FitPlan(batch, params, target, settings)
    runner = GraphStep(plan) if graph else None
    history = {"iter": [], "psnr": [], "replans": 0, "tuned": tuned}
    snap = plan.state() if settings.deterministic else None
    done = 0
    while done < iters:
        chunk = min(check_every if check_every > 0 else iters, iters - done)
        for k in range(chunk):
            if runner:
                runner.replay()
            else:
                plan.step()
            it = done + k + 1
            if log_every and it % log_every == 0:
                mse = plan.loss[:, 1].tolist()
                history["iter"].append(it)
                history["psnr"].append([psnr_from_mse(m) for m in mse])
        if plan.overflowed():
            history["replans"] += 1
            if settings.deterministic:
                plan.restore(snap)
            new_cap = plan.measure_entries() * 2 + 4096
            plan = _replan(plan, new_cap)
            runner = GraphStep(plan) if graph else None
            if settings.deterministic:  # redo this chunk with room for every entry
                keep = [i for i, it in enumerate(history["iter"]) if it <= done]
                history["iter"] = [history["iter"][i] for i in keep]
                history["psnr"] = [history["psnr"][i] for i in keep]
                continue
        done += chunk
        if settings.deterministic:
            snap = plan.state()
    image, loss = plan.render()
    history["final_psnr"] = [psnr_from_mse(m) for m in loss[:, 1].tolist()]
    history["images"] = batch.split_images(image)
    # write the fitted values back into the caller's per-image tensors
    for b, f in enumerate(fields):
        sl = batch.gaussian_slice(b)
        for k in PARAM_NAMES:
            if f.get(k) is not None:
                f[k].copy_(params[k][sl])
    history["plan"] = plan
    return history


def _replan(plan: FitPlan, capacity: int) -> FitPlan:
    new = FitPlan(plan.batch, plan.params, plan.target, plan.s, capacity=capacity)
    for k in plan.exp_avg:
        new.exp_avg[k].copy_(plan.exp_avg[k])
        new.exp_avg_sq[k].copy_(plan.exp_avg_sq[k])
    new.step_state.copy_(plan.step_state)
    return new
