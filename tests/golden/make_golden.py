"""Generate the golden vectors that pin the oracle to the reference implementation.

Run in a container where the reference source tree is available::

    python tests/golden/make_golden.py --reference-src <reference>/src

It imports the reference's own modules (``structsplat.render``, ``gaussians``,
``cuda_render._build_tile_index``, ``structure_tensor``), runs them on small seeded inputs and
writes ``tests/golden/*.npz``.  The tests then check the CPU oracle — and, on a GPU host, the
CUDA library — against these vectors; the reference itself is not needed at test time.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


def _field(ref, seed, N, H, W, lo, hi, spread, opac_range=None, elongated=False):
    import torch  # noqa: F401
    rng = np.random.default_rng(seed)
    means = np.stack([rng.uniform(-spread, W + spread, N), rng.uniform(-spread, H + spread, N)], 1)
    if elongated:
        sx = np.exp(rng.uniform(np.log(2.0), np.log(8.0), N))
        sy = np.exp(rng.uniform(np.log(0.5), np.log(1.2), N))
        scales = np.stack([sx, sy], 1)
    else:
        scales = np.exp(rng.uniform(np.log(lo), np.log(hi), (N, 2)))
    angles = rng.uniform(0, np.pi, N)
    colors = rng.random((N, 3))
    logits = None
    if opac_range is not None:
        o = rng.uniform(opac_range[0], opac_range[1], N)
        logits = np.log(o) - np.log1p(-o)
    g = ref.gaussians.GaussianField.from_numpy(means, scales, angles, colors, opacities=logits)
    return g


def render_case(ref, name, g, H, W, *, normalize, use_opacity, dilation, fade_alpha,
                sigma_cutoff=3.0, eps=1e-8, seed=0):
    """Forward image + gradients (w.r.t. render inputs and RS params), float32 and float64."""
    import torch
    out = {"H": H, "W": W, "normalize": int(normalize), "dilation": dilation,
           "fade_alpha": fade_alpha, "sigma_cutoff": sigma_cutoff, "eps": eps,
           "use_opacity": int(use_opacity)}
    rng = np.random.default_rng(1000 + seed)
    grad_out = rng.normal(0.0, 1.0, (H, W, 3))
    out["grad_out"] = grad_out.astype(np.float32)
    mode = "normalized" if normalize else "additive"
    for dt, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        means = g.means.detach().to(dt).clone()
        log_scales = g.log_scales.detach().to(dt).clone()
        rot = g.rotations.detach().to(dt).clone()
        colors = g.colors.detach().to(dt).clone()
        logits = None if (g.opacities is None or not use_opacity) else g.opacities.detach().to(dt).clone()
        field = ref.gaussians.GaussianField(means, log_scales, rot, colors, logits).trainable()
        conics = field.conics(dilation)
        radii = field.radii(sigma_cutoff, dilation)
        opac = field.opacity_values()
        if tag == "f32":
            out["means"] = means.detach().numpy().astype(np.float32)
            out["log_scales"] = log_scales.detach().numpy().astype(np.float32)
            out["rotations"] = rot.detach().numpy().astype(np.float32)
            out["colors"] = colors.detach().numpy().astype(np.float32)
            out["conics"] = conics.detach().numpy().astype(np.float32)
            out["radii"] = radii.numpy().astype(np.int64)
            if opac is not None:
                out["opacity_logits"] = logits.detach().numpy().astype(np.float32)
                out["opacities"] = opac.detach().numpy().astype(np.float32)
        # gradients w.r.t. the render inputs (conics and opacities as leaves)
        c_leaf = conics.detach().clone().requires_grad_(True)
        o_leaf = None if opac is None else opac.detach().clone().requires_grad_(True)
        m_leaf = means.detach().clone().requires_grad_(True)
        col_leaf = colors.detach().clone().requires_grad_(True)
        img = ref.render.render_field(m_leaf, c_leaf, col_leaf, radii, H, W, mode=mode,
                                      opacities=o_leaf, support_fade=fade_alpha > 0,
                                      sigma_cutoff=sigma_cutoff, support_fade_alpha=fade_alpha,
                                      normalization_eps=eps)
        go = torch.as_tensor(grad_out, dtype=dt)
        leaves = [m_leaf, c_leaf, col_leaf] + ([o_leaf] if o_leaf is not None else [])
        grads = torch.autograd.grad(img, leaves, go, allow_unused=True)
        out[f"image_{tag}"] = img.detach().numpy()
        for key, gr, leaf in zip(["g_means", "g_conics", "g_colors", "g_opacities"], grads, leaves):
            out[f"{key}_{tag}"] = (torch.zeros_like(leaf) if gr is None else gr).numpy()
        # gradients through the RS parameterisation (what a fit iteration differentiates)
        img2 = ref.render.render_field(field.means, conics, field.colors, radii, H, W, mode=mode,
                                       opacities=opac, support_fade=fade_alpha > 0,
                                       sigma_cutoff=sigma_cutoff, support_fade_alpha=fade_alpha,
                                       normalization_eps=eps)
        params = [field.means, field.log_scales, field.rotations, field.colors]
        if field.opacities is not None:
            params.append(field.opacities)
        pg = torch.autograd.grad(img2, params, go, allow_unused=True)
        for key, gr, p in zip(["rs_means", "rs_log_scales", "rs_rotations", "rs_colors",
                               "rs_opacity_logits"], pg, params):
            out[f"{key}_{tag}"] = (torch.zeros_like(p) if gr is None else gr).detach().numpy()
    np.savez_compressed(HERE / f"render_{name}.npz", **out)
    return out


def streamed_cases(ref):
    """A 96×96 cut of the heavy-tailed stress field (σ = exp(N(ln 2, 1.2)), 30 % elongated with
    aspect U[5, 50]) with 3,500 Gaussians: every 16- and 32-px tile list holds 531–1,411
    Gaussians, more than the CUDA kernels stage at once, and 911 rectangles are wider than
    48 px — the fixture that takes the streamed kernel paths to the reference's own result."""
    from structsplat_b200.synthetic import make_stress_field
    H = W = 96
    angle = np.random.default_rng(8).uniform(0, np.pi, (H, W)).astype(np.float32)
    f = make_stress_field(H, W, 3500, seed=9, along_edge_angle=angle)
    g = ref.gaussians.GaussianField.from_numpy(f.means, np.exp(f.log_scales), f.rotations,
                                               f.colors, opacities=f.opacity_logits)
    render_case(ref, "streamed_96_3500", g, H, W, normalize=True, use_opacity=True,
                dilation=0.0, fade_alpha=0.0, seed=60)
    render_case(ref, "streamed_96_3500_additive", g, H, W, normalize=False, use_opacity=True,
                dilation=0.0, fade_alpha=0.0, seed=61)


def tile_case(ref, name, means, radii, H, W, ts):
    import torch
    m = torch.as_tensor(np.asarray(means, np.float32))
    r = torch.as_tensor(np.asarray(radii, np.int64))
    gids, offsets = ref.cuda_render._build_tile_index(m, r, H, W, ts)
    off = offsets.numpy()
    gid = gids.numpy()
    sets = np.concatenate([np.sort(gid[off[t]:off[t + 1]]) for t in range(len(off) - 1)]) \
        if gid.size else np.zeros(0, np.int64)
    np.savez_compressed(HERE / f"tile_{name}.npz", means=m.numpy(), radii=r.numpy(), H=H, W=W,
                        tile_size=ts, offsets=off.astype(np.int64), gids_sorted=sets.astype(np.int64))


def structure_case(ref, name, img, **cfg):
    cfg_obj = ref.config.StructureTensorConfig(**cfg)
    t = ref.structure_tensor.compute(img, cfg_obj)
    np.savez_compressed(
        HERE / f"st_{name}.npz", img=img.astype(np.float32),
        grad_sigma=cfg_obj.grad_sigma, tensor_sigma=cfg_obj.tensor_sigma,
        gradient_operator=cfg_obj.gradient_operator, color_space=cfg_obj.color_space,
        flat_frac=cfg_obj.flat_frac, corner_frac=cfg_obj.corner_frac,
        lam1=t.lam1, lam2=t.lam2, angle=t.across_edge_angle, coherence=t.coherence,
        energy=t.energy, label=t.label, energy_ref=t.energy_ref)


def placement_cases(ref, make_target):
    """density_from_energy, sample_candidates and build_field (density_random) fixtures."""
    scfg = ref.config.StructureTensorConfig(grad_sigma=1.0, tensor_sigma=2.0)
    img = make_target(40, 48, seed=12)
    t = ref.structure_tensor.compute(img, scfg)
    for k, (base, power) in enumerate(((0.05, 1.0), (0.2, 2.0), (0.0, 0.5), (0.1, 1.7))):
        d = ref.density.density_from_energy(t.energy, base, power, t.energy_ref)
        np.savez_compressed(HERE / f"pl_density_{k}.npz", energy=t.energy, ref=t.energy_ref,
                            base=base, power=power, density=d)
    d = ref.density.density_from_energy(np.zeros((6, 7), np.float32), 0.0, 1.0, 1.0)
    np.savez_compressed(HERE / "pl_density_flat.npz", energy=np.zeros((6, 7), np.float32),
                        ref=1.0, base=0.0, power=1.0, density=d)
    d = ref.density.density_from_energy(t.energy, 0.05, 1.0, t.energy_ref)
    for seed, n in ((3, 500), (4, 3000)):
        pts = ref.density.sample_candidates(d, n, np.random.default_rng(seed))
        np.savez_compressed(HERE / f"pl_sample_{seed}.npz", density=d, n=n, seed=seed,
                            points=pts)
    for strategy, n, seed in (("aniso_onedge", 800, 5), ("iso_blue_noise", 600, 6)):
        icfg = ref.config.InitConfig(strategy=strategy, sampling_mode="density_random",
                                     num_gaussians=n, seed=seed)
        g = ref.init.build_field(img, icfg, scfg)
        np.savez_compressed(
            HERE / f"pl_field_{strategy}.npz", img=img, n=n, seed=seed,
            anisotropic=int(strategy == "aniso_onedge"), energy=t.energy,
            energy_ref=t.energy_ref, angle=t.across_edge_angle, coherence=t.coherence,
            density=d, means=g.means.detach().numpy(), log_scales=g.log_scales.detach().numpy(),
            rotations=g.rotations.detach().numpy(), colors=g.colors.detach().numpy())


def passes_cases(ref):
    """gaussian_activity and _raw_weight_map_field fixtures (render.py:417-442, fit.py:338-367)."""
    import torch
    H, W = 30, 34
    for name, alpha, seed in (("plain", 0.0, 61), ("fade", 1.0, 62), ("frac", 0.5, 63)):
        g = _field(ref, seed, 40, H, W, 0.6, 5.0, 4.0, opac_range=(0.2, 1.0))
        conics = g.conics()
        radii = g.radii(3.0)
        act = ref.render.gaussian_activity(g.means.detach(), conics.detach(), radii, H, W,
                                           support_fade=alpha > 0, support_fade_alpha=alpha)
        cfg = ref.config.FitConfig(support_fade=alpha > 0)
        g.trainable()
        den = ref.fit._raw_weight_map_field(g, cfg, H, W, support_fade_alpha=alpha)
        G = torch.as_tensor(np.random.default_rng(seed).normal(size=H * W), dtype=den.dtype)
        params = [g.means, g.log_scales, g.rotations, g.opacities]
        grads = torch.autograd.grad((den * G).sum(), params)
        np.savez_compressed(
            HERE / f"pass_{name}.npz", H=H, W=W, fade_alpha=alpha,
            means=g.means.detach().numpy(), log_scales=g.log_scales.detach().numpy(),
            rotations=g.rotations.detach().numpy(), opacity_logits=g.opacities.detach().numpy(),
            conics=conics.detach().numpy(), radii=radii.numpy(), activity=act.numpy(),
            den=den.detach().numpy(), G=G.numpy(),
            **{f"g_{k}": v.numpy() for k, v in zip(
                ("means", "log_scales", "rotations", "opacity_logits"), grads)})


def fit_case(ref, make_field, make_target):
    """The plain fit of the CPU benchmark case (256², 4,096 Gaussians, 100 Adam steps at lr 1e-2,
    pixel MSE, normalized renderer) with the reference's own modules: render_field, the field's
    parameter groups in torch.optim.Adam, and the post-step log-scale clamp (fit.py:3033,
    3359-3366).  Records the PSNR of the pre-step render every 10 steps and after the last."""
    import math
    import torch
    H = W = 256
    f = make_field(H, W, 4096, seed=71)
    target = torch.as_tensor(make_target(H, W, seed=72))
    g = ref.gaussians.GaussianField(*[torch.as_tensor(getattr(f, k)).clone() for k in
                                      ("means", "log_scales", "rotations", "colors",
                                       "opacity_logits")]).trainable()
    opt = torch.optim.Adam(g.parameter_groups(1e-2, 1e-2, 1e-2, 1e-2, 1e-2))
    lo, hi = math.log(0.35), math.log(max(H, W))
    psnr = []

    def render():
        return ref.render.render_field(g.means, g.conics(), g.colors, g.radii(3.0), H, W,
                                       mode="normalized", opacities=g.opacity_values())
    for it in range(100):
        img = render()
        loss = ((img - target) ** 2).mean(dim=2).mean()
        if it % 10 == 0:
            psnr.append(10 * math.log10(1.0 / float(((img.detach() - target) ** 2).mean())))
        opt.zero_grad(set_to_none=True)
        loss.backward()
        opt.step()
        with torch.no_grad():
            g.log_scales.clamp_(max=hi)
            g.log_scales.clamp_(min=lo)
    with torch.no_grad():
        img = render()
    psnr.append(10 * math.log10(1.0 / float(((img - target) ** 2).mean())))
    np.savez_compressed(HERE / "fit_plain_256_4096.npz", seed_field=71, seed_target=72,
                        psnr=np.array(psnr), **{k: getattr(g, a).detach().numpy() for k, a in (
                            ("means", "means"), ("log_scales", "log_scales"),
                            ("rotations", "rotations"), ("colors", "colors"),
                            ("opacity_logits", "opacities"))})


def codec_cases(ref, make_field, make_target):
    """SSPL1 containers written by the reference's codec.encode, with its decode and
    decode_and_render results (codec.py:235-500)."""
    import torch
    H, W = 48, 64
    cases = [
        ("default_opacity", dict(), True, False),
        ("plain_noopacity", dict(morton_reorder=False, color_delta=False,
                                 means_byte_planar=False, rot_circular=False, bits_means=12,
                                 bits_scales=10, bits_rot=9, bits_colors=7), False, False),
        ("png_alpha", dict(stream_codec="png", bits_opacity=6), True, True),
    ]
    for k, (name, kw, with_opacity, with_alpha) in enumerate(cases):
        f = make_field(H, W, 400, seed=81 + k)
        g = ref.gaussians.GaussianField(
            torch.as_tensor(f.means), torch.as_tensor(f.log_scales), torch.as_tensor(f.rotations),
            torch.as_tensor(f.colors),
            torch.as_tensor(f.opacity_logits) if with_opacity else None)
        alpha = make_target(H, W, seed=90 + k)[..., 0] if with_alpha else None
        blob = ref.codec.encode(g, H, W, ref.codec.CodecConfig(**kw), alpha=alpha)
        d = ref.codec.decode(blob)
        img = ref.codec.decode_and_render(blob)
        out = dict(blob=np.frombuffer(blob, dtype=np.uint8), H=H, W=W,
                   means=d.means.numpy(), log_scales=d.log_scales.numpy(),
                   rotations=d.rotations.numpy(), colors=d.colors.numpy(),
                   image=img.detach().numpy())
        if d.opacities is not None:
            out["opacity_logits"] = d.opacities.numpy()
        a = ref.codec.decode_alpha(blob)
        if a is not None:
            out["alpha"] = a
        np.savez_compressed(HERE / f"codec_{name}.npz", **out)


def ssim_cases(ref, make_target):
    """The SSIM term of the fit loss (metrics.py:130-150) and its mix with the L1 pixel loss
    (fit.py:3244): value and gradient w.r.t. the rendered image, from the reference's own
    metrics.ssim and fit._pixel_loss under torch autograd."""
    import torch
    M = ref.metrics
    for name, (H, W, seed, w) in {"ssim_small": (23, 31, 3, 0.3), "ssim_tiny": (7, 5, 4, 0.3),
                                  "ssim_square": (40, 40, 5, 0.8)}.items():
        target = torch.tensor(make_target(H, W, seed=seed))
        rng = np.random.default_rng(seed + 100)
        pred0 = np.clip(target.numpy() + rng.normal(0, 0.15, target.shape), 0, 1)
        pred = torch.tensor(pred0.astype(np.float32), requires_grad=True)
        s = M.ssim(pred, target)
        (g_ssim,) = torch.autograd.grad(s, pred)
        pred2 = torch.tensor(pred0.astype(np.float32), requires_grad=True)
        stats = M.SSIMTargetStats(target)
        s_cached = M.ssim(pred2, target, target_stats=stats)
        pix = ref.fit._pixel_loss(pred2, target, "l1")
        loss = (1 - w) * pix + w * (1 - s_cached)
        (g_loss,) = torch.autograd.grad(loss, pred2)
        np.savez(HERE / f"{name}.npz", pred=pred0.astype(np.float32), target=target.numpy(),
                 weight=np.float32(w), ssim=np.float32(s.item()),
                 ssim_cached=np.float32(s_cached.item()), grad_ssim=g_ssim.numpy(),
                 loss=np.float32(loss.item()), grad_loss=g_loss.numpy())


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-src", required=True,
                    help="the reference project's src directory (holding structsplat/)")
    ap.add_argument("--only", choices=["placement", "passes", "fit", "codec", "ssim",
                                       "streamed"],
                    default=None,
                    help="regenerate one group of fixtures, leaving the others untouched")
    args = ap.parse_args()
    sys.path.insert(0, args.reference_src)
    sys.path.insert(0, str(REPO))
    import torch
    import structsplat.codec
    import structsplat.config
    import structsplat.cuda_render
    import structsplat.density
    import structsplat.fit
    import structsplat.gaussians
    import structsplat.init
    import structsplat.metrics
    import structsplat.render
    import structsplat.structure_tensor

    from structsplat_b200.synthetic import make_field, make_target

    class Ref:
        codec = structsplat.codec
        config = structsplat.config
        cuda_render = structsplat.cuda_render
        density = structsplat.density
        fit = structsplat.fit
        gaussians = structsplat.gaussians
        init = structsplat.init
        metrics = structsplat.metrics
        render = structsplat.render
        structure_tensor = structsplat.structure_tensor

    torch.manual_seed(0)
    if args.only == "streamed":
        for old in HERE.glob("render_streamed_*.npz"):
            old.unlink()
        streamed_cases(Ref)
        print("wrote", len(list(HERE.glob("render_streamed_*.npz"))), "streamed render fixtures")
        return
    if args.only == "ssim":
        for old in HERE.glob("ssim_*.npz"):
            old.unlink()
        ssim_cases(Ref, make_target)
        print("wrote", len(list(HERE.glob("ssim_*.npz"))), "ssim fixtures")
        return
    if args.only == "codec":
        for old in HERE.glob("codec_*.npz"):
            old.unlink()
        codec_cases(Ref, make_field, make_target)
        print("wrote", len(list(HERE.glob("codec_*.npz"))), "codec fixtures")
        return
    if args.only == "fit":
        fit_case(Ref, make_field, make_target)
        print("wrote the fit fixture")
        return
    if args.only == "passes":
        for old in HERE.glob("pass_*.npz"):
            old.unlink()
        passes_cases(Ref)
        print("wrote", len(list(HERE.glob("pass_*.npz"))), "pass fixtures")
        return
    if args.only == "placement":
        for old in HERE.glob("pl_*.npz"):
            old.unlink()
        placement_cases(Ref, make_target)
        print("wrote", len(list(HERE.glob("pl_*.npz"))), "placement fixtures")
        return
    for old in HERE.glob("*.npz"):
        old.unlink()

    # --- tile index -------------------------------------------------------------------
    tile_case(Ref, "known_answer", [[2.0, 2.0], [20.0, 20.0]], [[1, 1], [1, 1]], 8, 8, 4)
    rng = np.random.default_rng(21)
    N, H, W = 40, 33, 29
    g = _field(Ref, 21, N, H, W, 0.6, 6.0, 4.0)
    tile_case(Ref, "elongated_ts8", g.means.detach().numpy(), g.radii(3.0).numpy(), H, W, 8)
    f = make_field(90, 100, 300, seed=5)
    gf = Ref.gaussians.GaussianField(torch.as_tensor(f.means), torch.as_tensor(f.log_scales),
                                     torch.as_tensor(f.rotations), torch.as_tensor(f.colors))
    tile_case(Ref, "synthetic_ts16", f.means, gf.radii(3.0).numpy(), 90, 100, 16)
    tile_case(Ref, "synthetic_ts4", f.means, gf.radii(3.0).numpy(), 90, 100, 4)
    # The reference's torch builder has no non-finite guard (its CUDA kernel drops non-finite
    # centres, render_ext.cu:25-34); far-away and half-way centres are pinned here.
    tile_case(Ref, "far_and_ties_ts4", [[5.0, 5.0], [1e12, 1e12], [-1e12, 4.0], [2.5, 3.5],
                                        [11.49, -0.5], [-3.5, 6.5]],
              [[2, 2], [2, 2], [2, 2], [1, 3], [0, 1], [4, 1]], 12, 12, 4)
    del rng

    # --- renderer --------------------------------------------------------------------
    k = 0
    for normalize in (True, False):
        for use_opacity in (False, True):
            for dilation in (0.0, 0.3):
                for fade in (0.0, 1.0):
                    g = _field(Ref, 7, 20, 16, 18, 0.7, 3.5, 2.0,
                               opac_range=(0.1, 1.0) if use_opacity else None)
                    name = (f"matrix_{'norm' if normalize else 'add'}_{'op' if use_opacity else 'noop'}"
                            f"_d{int(dilation * 10)}_f{int(fade)}")
                    render_case(Ref, name, g, 16, 18, normalize=normalize,
                                use_opacity=use_opacity, dilation=dilation, fade_alpha=fade,
                                seed=k)
                    k += 1
    g = _field(Ref, 11, 32, 21, 23, 0.7, 4.0, 3.0, opac_range=(0.2, 1.0))
    render_case(Ref, "tiled_fade_opacity", g, 21, 23, normalize=True, use_opacity=True,
                dilation=0.0, fade_alpha=1.0, seed=50)
    g = _field(Ref, 22, 48, 40, 44, 0.5, 8.0, 3.0, elongated=True)
    render_case(Ref, "elongated_fade", g, 40, 44, normalize=True, use_opacity=False,
                dilation=0.0, fade_alpha=1.0, seed=51)
    g = _field(Ref, 4, 12, 16, 17, 0.8, 3.0, 2.0, opac_range=(0.2, 0.9))
    render_case(Ref, "fractional_fade", g, 16, 17, normalize=True, use_opacity=True,
                dilation=0.0, fade_alpha=0.5, seed=52)
    g = _field(Ref, 23, 37, 23, 25, 0.7, 4.0, 2.0, opac_range=(0.27, 0.73))
    render_case(Ref, "eps_1e-6_additive_check", g, 23, 25, normalize=True, use_opacity=True,
                dilation=0.0, fade_alpha=0.0, eps=1e-6, seed=53)
    f = make_field(64, 64, 256, seed=3)
    gf = Ref.gaussians.GaussianField.from_numpy(f.means, np.exp(f.log_scales), f.rotations,
                                                f.colors, opacities=f.opacity_logits)
    render_case(Ref, "synthetic_64_256", gf, 64, 64, normalize=True, use_opacity=True,
                dilation=0.0, fade_alpha=0.0, seed=54)
    render_case(Ref, "synthetic_64_256_additive", gf, 64, 64, normalize=False, use_opacity=True,
                dilation=0.0, fade_alpha=0.0, seed=55)
    g = Ref.gaussians.GaussianField.from_numpy(np.array([[25.0, 5.0]]), np.array([[10.0, 10.0]]),
                                               np.zeros(1), np.array([[1.0, 0.0, 0.0]]))
    render_case(Ref, "offimage", g, 10, 10, normalize=True, use_opacity=False, dilation=0.0,
                fade_alpha=0.0, seed=56)
    # Far-away centre (the reference CUDA path also drops NaN centres; the torch path cannot
    # take them, so the NaN contract is checked against the oracle's empty-support rule).
    g = Ref.gaussians.GaussianField.from_numpy(np.array([[5.0, 5.0], [1e12, 1e12], [7.5, 2.5]]),
                                               np.full((3, 2), 1.5), np.zeros(3), np.ones((3, 3)))
    render_case(Ref, "far_away", g, 12, 12, normalize=True, use_opacity=False, dilation=0.0,
                fade_alpha=0.0, seed=57)
    streamed_cases(Ref)

    # --- structure tensor ------------------------------------------------------------
    edge = np.zeros((64, 64, 3), np.float32)
    edge[:, 32:, :] = 1.0
    for op in ("central", "sobel", "scharr"):
        structure_case(Ref, f"edge_{op}", edge, gradient_operator=op)
    structure_case(Ref, "edge_rgb", edge, color_space="rgb")
    noise = np.clip(0.5 + 0.01 * np.random.default_rng(0).standard_normal((64, 64, 3)), 0, 1)
    structure_case(Ref, "noise", noise.astype(np.float32))
    iso = np.zeros((32, 32, 3), np.float32)
    iso[:, :16] = [1.0, 0.0, 0.0]
    iso[:, 16:] = [0.0, 0.2126 / 0.7152, 0.0]
    structure_case(Ref, "isoluminant_rgb", iso, color_space="rgb")
    tgt = make_target(48, 40, seed=9)
    structure_case(Ref, "synthetic_rho2", tgt, grad_sigma=1.0, tensor_sigma=2.0)
    structure_case(Ref, "synthetic_rho3", tgt, grad_sigma=1.0, tensor_sigma=3.0)
    structure_case(Ref, "synthetic_rgb_rho2", tgt, grad_sigma=1.0, tensor_sigma=2.0,
                   color_space="rgb")
    structure_case(Ref, "tiny_5x3", make_target(5, 3, seed=4), grad_sigma=1.0, tensor_sigma=2.0)
    placement_cases(Ref, make_target)
    passes_cases(Ref)
    fit_case(Ref, make_field, make_target)
    codec_cases(Ref, make_field, make_target)
    ssim_cases(Ref, make_target)
    print("wrote", len(list(HERE.glob("*.npz"))), "fixtures")


if __name__ == "__main__":
    main()
