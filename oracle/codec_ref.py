"""CPU oracle of the SSPL1 field decode (test infrastructure only).

Restates ``src/structsplat/codec.py:80-131,333-391`` in NumPy: container framing, stream
inflate (zlib; PNG through Pillow), unpacking (byte-planar for the means), the modular prefix
sums that undo the Morton-order and colour deltas, and float64 dequantisation.  Pinned by the
``codec_*`` fixtures written with the reference's own encoder and decoder.
"""
from __future__ import annotations

import json
import struct
import zlib
from io import BytesIO

import numpy as np


def _item(bits):
    return np.dtype(np.uint8 if bits <= 8 else (np.uint16 if bits <= 16 else np.uint32))


def _unpack(raw, bits, count, planar=False):
    dt = _item(bits)
    if planar and dt.itemsize > 1:
        planes = np.frombuffer(raw, np.uint8, count=count * dt.itemsize).reshape(dt.itemsize, count)
        return np.frombuffer(np.ascontiguousarray(planes.T).tobytes(), dt, count=count).astype(
            np.uint32)
    return np.frombuffer(raw, dt, count=count).astype(np.uint32)


def _dequant(q, lo, hi, bits):
    levels = (1 << bits) - 1
    return (lo + (q.astype(np.float64) / levels) * (np.asarray(hi) - lo)).astype(np.float32)


def _inflate(payload, codec, raw_len):
    if codec == "zlib":
        return zlib.decompress(payload)
    from PIL import Image
    arr = np.asarray(Image.open(BytesIO(payload)).convert("L"), dtype=np.uint8).reshape(-1)
    return arr[:raw_len].tobytes()


def decode(blob: bytes) -> dict:
    assert blob[:5] == b"SSPL1"
    (hlen,) = struct.unpack_from("<I", blob, 5)
    h = json.loads(blob[9:9 + hlen])
    off = 9 + hlen
    n, H, W = h["n"], h["H"], h["W"]
    bm, bs, br, bc = h["bits"]
    has_op = bool(h.get("has_opacity", False))
    lens = h.get("stream_raw_lengths", [])
    raws = []
    for i in range(5 if has_op else 4):
        (zlen,) = struct.unpack_from("<I", blob, off)
        off += 4
        raws.append(_inflate(blob[off:off + zlen], h.get("stream_codec", "zlib"),
                             int(lens[i]) if i < len(lens) else None))
        off += zlen
    qm = _unpack(raws[0], bm, 2 * n, h.get("means_byte_planar", False)).reshape(2, n).T
    if h["morton"]:
        qm = np.cumsum(qm, axis=0, dtype=np.uint64).astype(np.uint32) & ((1 << bm) - 1)
    qs = _unpack(raws[1], bs, 2 * n).reshape(2, n).T
    qr = _unpack(raws[2], br, n)
    qc = _unpack(raws[3], bc, 3 * n).reshape(3, n).T
    if h.get("color_delta", False):
        qc = np.cumsum(qc, axis=0, dtype=np.uint64).astype(np.uint32) & ((1 << bc) - 1)
    out = {"means": _dequant(qm, h.get("means_lo", [0.0, 0.0]),
                             h.get("means_hi", [W - 1.0, H - 1.0]), bm),
           "log_scales": _dequant(qs, h.get("scale_lo", [float(np.log(0.35))] * 2),
                                  h.get("scale_hi", [float(np.log(max(H, W)))] * 2), bs),
           "rotations": ((qr.astype(np.float64) / (1 << br)) * np.pi).astype(np.float32)
           if h.get("rot_circular", False) else _dequant(qr, 0.0, np.pi, br),
           "colors": _dequant(qc, np.asarray(h["color_lo"]), np.asarray(h["color_hi"]), bc)}
    if has_op:
        b = h["bits_opacity"]
        p = _dequant(_unpack(raws[4], b, n), 0.0, 1.0, b).clip(1e-4, 1.0 - 1e-4)
        out["opacity_logits"] = np.log(p / (1.0 - p)).astype(np.float32)
    return out
