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
