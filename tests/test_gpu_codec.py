"""SSPL1 decode → render on the GPU against the reference's decode and decode_and_render.

Bars: decoded means, log-scales, rotations and colours bit-identical; opacity logits within
2 ulp (CUDA logf vs numpy's float32 log); the rendered image within 1e-5 relative of the
reference's render of its own decoded field; alpha maps exact.
"""
from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import golden, golden_names
from gpu_helpers import rel_err, require_cuda
from structsplat_b200 import codec

pytestmark = pytest.mark.gpu
CASES = golden_names("codec_")


@pytest.mark.parametrize("name", CASES)
def test_decode_matches_reference(name):
    require_cuda()
    z = golden(name)
    blob = z["blob"].tobytes()
    f = codec.decode(blob)
    for k in ("means", "log_scales", "rotations", "colors"):
        assert np.array_equal(f[k].cpu().numpy(), z[k]), k
    if "opacity_logits" in z.files:
        got, want = f["opacity_logits"].cpu().numpy(), z["opacity_logits"]
        ulp = np.abs(got.view(np.int32).astype(np.int64) - want.view(np.int32).astype(np.int64))
        assert ulp.max() <= 2
    else:
        assert f["opacity_logits"] is None
    assert codec.blob_header(blob)["n"] == f["means"].shape[0]


@pytest.mark.parametrize("name", CASES)
def test_decode_and_render_matches_reference(name):
    require_cuda()
    z = golden(name)
    img = codec.decode_and_render(z["blob"].tobytes())
    assert rel_err(img, z["image"]) <= 1e-5


def test_alpha_stream():
    require_cuda()
    z = golden("codec_png_alpha.npz")
    a = codec.decode_alpha(z["blob"].tobytes())
    assert torch.equal(a.cpu(), torch.tensor(z["alpha"]))
    assert codec.decode_alpha(golden("codec_default_opacity.npz")["blob"].tobytes()) is None
