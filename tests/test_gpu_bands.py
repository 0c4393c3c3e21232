"""One image in bands of tile rows on the GPU (one process evaluates every band, as the ranks
would): the band images stack into the full image bitwise and the summed band gradients equal
the full image's RS gradients."""
from __future__ import annotations

import pytest
import torch

from gpu_helpers import rel_err, require_cuda
from structsplat_b200.bands import BandPlan, band_rows
from structsplat_b200.fit import RenderPlan
from structsplat_b200.synthetic import make_field

pytestmark = pytest.mark.gpu
NAMES = ("means", "log_scales", "rotations", "colors", "opacity_logits")


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("world", [2, 3])
def test_band_images_stack_and_band_gradients_sum(world, deterministic):
    require_cuda()
    H, W = 200, 150
    f = make_field(H, W, 3000, seed=13)
    params = {k: torch.tensor(getattr(f, k), device="cuda") for k in NAMES}
    go = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(4))
    full = RenderPlan.for_field(params, H, W, deterministic=deterministic)
    want = {k: v.clone() for k, v in full.forward_backward(params, go).items()}
    want_img = full.image.view(H, W, 3).clone()
    images, total = [], None
    for r in range(world):
        y0, y1 = band_rows(H, W, r, world)
        band = BandPlan(params, H, W, y0, y1, deterministic=deterministic)
        img, grads = band.forward_backward(params, go)
        images.append(img.clone())
        total = ({k: v.clone() for k, v in grads.items()} if total is None
                 else {k: total[k] + grads[k] for k in total})
    assert torch.equal(torch.cat(images, 0), want_img)
    for k in want:
        assert rel_err(total[k], want[k]) <= 1e-5, k


def test_bands_stack_bitwise_for_centres_one_ulp_above_half_integers():
    """Centres 1 ulp above half-integers round up in the full image's support rectangles; a band
    that shifted its means by the band origin would round some of them the other way.  The
    bands keep image coordinates, so they stack bitwise all the same."""
    require_cuda()
    import numpy as np
    H, W = 160, 96
    f = make_field(H, W, 2000, seed=21)
    my = np.floor(f.means[:, 1]).astype(np.float32) + np.float32(0.5)
    f.means[:, 1] = np.nextafter(my, np.float32(np.inf))
    params = {k: torch.tensor(getattr(f, k), device="cuda") for k in NAMES}
    go = torch.randn(H, W, 3, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
    full = RenderPlan.for_field(params, H, W, deterministic=True)
    want = {k: v.clone() for k, v in full.forward_backward(params, go).items()}
    want_img = full.image.view(H, W, 3).clone()
    images, total = [], None
    for r in range(4):
        y0, y1 = band_rows(H, W, r, 4)
        band = BandPlan(params, H, W, y0, y1, deterministic=True)
        img, grads = band.forward_backward(params, go)
        images.append(img.clone())
        total = ({k: v.clone() for k, v in grads.items()} if total is None
                 else {k: total[k] + grads[k] for k in total})
    assert torch.equal(torch.cat(images, 0), want_img)
    for k in want:
        assert rel_err(total[k], want[k]) <= 1e-5, k
