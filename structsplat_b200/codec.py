"""SSPL1 container decode → render on the GPU (the decode step after fitting).

Mirrors ``structsplat.codec`` (codec.py:333-500): ``blob_header``, ``decode``,
``decode_alpha`` and ``decode_and_render`` take the same bytes and return the same field and
image.  The container is parsed and its streams inflated on the host (zlib, or PNG through
Pillow — serial byte codecs), the raw integer streams are uploaded once, and one library call
unpacks, undoes the Morton / colour deltas (prefix sums) and dequantises them on the device
(``ss_sspl1_dequantize``).  Rendering uses the semantics stored in the header (renderer,
dilation, σ cutoff, support fade, ε) through ``render_gaussians``.
"""
from __future__ import annotations

import ctypes
import json
import struct
import zlib
from io import BytesIO

import numpy as np
import torch

from . import _native
from .render import ADDITIVE_MODES, DEFAULT_EPS, NORMALIZED_MODES, _p, _stream

MAGIC = b"SSPL1"
SCALE_LO = float(np.log(0.35))  # the fitter's log-scale floor, for headers without scale_lo


def blob_header(blob: bytes) -> dict:
    """The JSON header of an SSPL1 container (codec.py:422-426)."""
    if len(blob) < 9 or blob[:5] != MAGIC:
        raise ValueError("not a structsplat codec blob")
    (hlen,) = struct.unpack_from("<I", blob, 5)
    return json.loads(blob[9:9 + hlen])


def _inflate(payload: bytes, codec: str, raw_len):
    if codec == "zlib":
        return zlib.decompress(payload)
    if codec == "png":
        if raw_len is None:
            raise ValueError("PNG stream requires stream_raw_lengths in the codec header")
        from PIL import Image
        arr = np.asarray(Image.open(BytesIO(payload)).convert("L"), dtype=np.uint8).reshape(-1)
        if arr.size < raw_len:
            raise ValueError(f"PNG stream too short: got {arr.size} bytes, expected {raw_len}")
        return arr[:raw_len].tobytes()
    raise ValueError(f"unknown stream_codec {codec!r}; expected 'zlib' or 'png'")


def _streams(blob: bytes):
    """(header, inflated stream bytes in container order)."""
    h = blob_header(blob)
    (hlen,) = struct.unpack_from("<I", blob, 5)
    off = 9 + hlen
    count = (5 if h.get("has_opacity", False) else 4) + (1 if h.get("has_alpha", False) else 0)
    raw_lengths = h.get("stream_raw_lengths", [])
    codec = h.get("stream_codec", "zlib")
    raws = []
    for i in range(count):
        if off + 4 > len(blob):
            raise ValueError("truncated structsplat codec stream framing")
        (zlen,) = struct.unpack_from("<I", blob, off)
        off += 4
        raw_len = int(raw_lengths[i]) if i < len(raw_lengths) else None
        raws.append(_inflate(blob[off:off + zlen], codec, raw_len))
        off += zlen
    return h, raws


def decode(blob: bytes, device="cuda") -> dict:
    """The field of an SSPL1 container as CUDA float32 tensors (means, log_scales, rotations,
    colors, opacity_logits or None), bit-identical to the reference's ``codec.decode`` except
    the opacity logit (within 2 ulp)."""
    h, raws = _streams(blob)
    n, H, W = int(h["n"]), int(h["H"]), int(h["W"])
    b_means, b_scales, b_rot, b_colors = (int(b) for b in h["bits"])
    has_opacity = bool(h.get("has_opacity", False))
    dev = torch.device(device)
    if dev.type != "cuda":
        raise RuntimeError("the B200 decoder requires a CUDA device")

    def up(raw):
        if not raw:
            return torch.zeros(1, dtype=torch.uint8, device=dev)
        return torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(dev)
    dev_raws = [up(r) for r in raws[:5 if has_opacity else 4]]
    s = _native.SsSspl1Streams()
    s.n = n
    s.means, s.scales, s.rotations, s.colors = (t.data_ptr() for t in dev_raws[:4])
    s.means_bits, s.scale_bits, s.rot_bits, s.color_bits = b_means, b_scales, b_rot, b_colors
    s.means_byte_planar = int(bool(h.get("means_byte_planar", False)))
    s.morton = int(bool(h["morton"]))
    s.rot_circular = int(bool(h.get("rot_circular", False)))
    s.color_delta = int(bool(h.get("color_delta", False)))
    means_lo = h.get("means_lo", [0.0, 0.0])
    means_hi = h.get("means_hi", [W - 1.0, H - 1.0])
    scale_lo = h.get("scale_lo", [SCALE_LO, SCALE_LO])
    scale_hi = h.get("scale_hi", [float(np.log(max(H, W)))] * 2)
    for d in range(2):
        s.means_lo[d], s.means_hi[d] = float(means_lo[d]), float(means_hi[d])
        s.scale_lo[d], s.scale_hi[d] = float(scale_lo[d]), float(scale_hi[d])
    for c in range(3):
        s.color_lo[c], s.color_hi[c] = float(h["color_lo"][c]), float(h["color_hi"][c])
    s.opacities = dev_raws[4].data_ptr() if has_opacity else None
    s.opacity_bits = int(h.get("bits_opacity", 8))
    f32 = dict(device=dev, dtype=torch.float32)
    field = {"means": torch.empty(n, 2, **f32), "log_scales": torch.empty(n, 2, **f32),
             "rotations": torch.empty(n, **f32), "colors": torch.empty(n, 3, **f32),
             "opacity_logits": torch.empty(n, **f32) if has_opacity else None}
    ws_bytes = _native.size_query("ss_sspl1_workspace_bytes", n)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    _native.call("ss_sspl1_dequantize", ctypes.byref(s), _p(field["means"]),
                 _p(field["log_scales"]), _p(field["rotations"]), _p(field["colors"]),
                 _p(field["opacity_logits"]), _p(ws), ws_bytes, _stream())
    return field


def decode_alpha(blob: bytes, device="cuda"):
    """The (H, W) float32 alpha map in [0, 1], or None for alpha-free blobs (codec.py:394-419)."""
    h, raws = _streams(blob)
    if not h.get("has_alpha", False):
        return None
    H, W = int(h["H"]), int(h["W"])
    # a true float32 division, as the reference computes it (a device division by a scalar
    # may multiply by its reciprocal instead, which rounds differently)
    a = np.frombuffer(raws[-1], dtype=np.uint8, count=H * W).reshape(H, W)
    return torch.from_numpy(a.astype(np.float32) / np.float32(255.0)).to(device)


def decode_and_render(blob: bytes, device="cuda", tile_size: int | None = None):
    """Decode and render with the header's render semantics (codec.py:482-500): (H, W, 3)."""
    from .field import render_gaussians
    from .render import RENDER_TILE
    h = blob_header(blob)
    f = decode(blob, device=device)
    H, W = int(h["H"]), int(h["W"])
    mode = h.get("renderer", "normalized")
    if mode in NORMALIZED_MODES:
        normalize = True
    elif mode in ADDITIVE_MODES:
        normalize = False
    else:
        raise ValueError(f"renderer {mode!r} is not supported by the B200 renderer")
    return render_gaussians(f["means"], f["log_scales"], f["rotations"], f["colors"], H, W,
                            opacity_logits=f["opacity_logits"], normalize=normalize,
                            eps=float(h.get("normalization_eps", DEFAULT_EPS)),
                            sigma_cutoff=float(h.get("sigma_cutoff", 3.0)),
                            dilation=float(h.get("aa_dilation", 0.0)),
                            support_fade=bool(h.get("support_fade", False)),
                            tile_size=tile_size or RENDER_TILE)
