"""ctypes binding of ``libstructsplat_b200.so`` (the C ABI in ``include/structsplat_b200.h``).

The library is built in-tree by ``structsplat_b200.build``.  There is no fallback: if the
library is missing or cannot be loaded, every entry point raises ``RuntimeError``.
"""
from __future__ import annotations

import collections
import ctypes
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libstructsplat_b200.so"

_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_f32 = ctypes.c_float
_f64 = ctypes.c_double
_szp = ctypes.POINTER(ctypes.c_size_t)


class SsBatch(ctypes.Structure):
    """``ss_batch`` of the C header: a batch of images rendered as one tile set."""
    _fields_ = [("images", ctypes.c_int), ("tile_size", ctypes.c_int),
                ("tiles", ctypes.c_int64), ("pixels", ctypes.c_int64),
                ("image_table", _vp), ("pixel_base", _vp), ("gaussian_base", _vp),
                ("gaussian_image", _vp), ("tile_image", _vp)]


class SsSspl1Streams(ctypes.Structure):
    """``ss_sspl1_streams`` of the C header."""
    _fields_ = [("n", ctypes.c_int64), ("means", _vp), ("means_bits", ctypes.c_int),
                ("means_byte_planar", ctypes.c_int), ("morton", ctypes.c_int),
                ("means_lo", _f64 * 2), ("means_hi", _f64 * 2), ("scales", _vp),
                ("scale_bits", ctypes.c_int), ("scale_lo", _f64 * 2), ("scale_hi", _f64 * 2),
                ("rotations", _vp), ("rot_bits", ctypes.c_int), ("rot_circular", ctypes.c_int),
                ("colors", _vp), ("color_bits", ctypes.c_int), ("color_delta", ctypes.c_int),
                ("color_lo", _f64 * 3), ("color_hi", _f64 * 3), ("opacities", _vp),
                ("opacity_bits", ctypes.c_int)]


_bp = ctypes.POINTER(SsBatch)
_pp = ctypes.POINTER(_vp)
_dp = ctypes.POINTER(_f64)

# name -> argtypes (all return int status unless listed in _RESTYPES)
SIGNATURES = {
    "ss_last_error": [],
    "ss_version": [],
    "ss_splat_record_bytes": [],
    "ss_pack_splats": [_vp, _vp, _vp, _vp, _vp, _i64, _int, _int, _vp, _vp],
    "ss_project_rs": [_vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _int, _int, _vp, _vp, _vp, _vp],
    "ss_project_rs_backward": [_vp, _vp, _vp, _i64, _f32, _vp, _vp, _vp, _vp, _vp, _vp],
    "ss_tile_index_workspace_bytes": [_i64, _int, _int, _int, _szp],
    "ss_tile_index_count": [_vp, _i64, _int, _int, _int, _int, _f32, _vp, _vp, ctypes.c_size_t,
                            _vp, _vp],
    "ss_tile_index_fill": [_vp, _i64, _int, _int, _int, _int, _f32, _vp, _vp, _i64, _vp,
                           ctypes.c_size_t, _vp, _vp],
    "ss_project_rs_index_count": [_vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _int, _int, _int,
                                  _int, _vp, _vp, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t,
                                  _vp, _vp],
    "ss_build_tile_index_static": [_vp, _vp, _vp, _i64, _int, _int, _int, _int, _f32, _vp, _i64,
                                   _vp, _vp, _vp],
    "ss_render_forward": [_vp, _i64, _vp, _i64, _vp, _int, _int, _int, _int, _f32, _f32, _vp, _vp,
                          _vp, _vp],
    "ss_set_backward_warps": [_int, _int],
    "ss_set_dependent_launch": [_int],
    "ss_get_dependent_launch": [],
    "ss_get_backward_warps": [_int],
    "ss_set_forward_chunk": [_int, _int],
    "ss_get_forward_chunk": [_int],
    "ss_render_backward_workspace_bytes": [_i64, _i64, _int, _int, _int, _szp],
    "ss_render_backward": [_vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _int, _int, _int, _int,
                           _f32, _f32, _int, _vp, _vp, _vp, _vp, _int, _vp, ctypes.c_size_t, _vp,
                           _vp],
    "ss_render_backward_moments": [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _int, _int,
                                   _int, _int, _f32, _f32, _int, _vp, ctypes.c_size_t, _vp, _vp],
    "ss_render_backward_finalize_rs": [_vp, _i64, _vp, _i64, _vp, _int, _int, _int, _int, _vp,
                                       _vp, _vp, _vp, _f32, _vp, _vp, _vp, _vp, _vp, _vp],
    "ss_gaussian_activity": [_vp, _i64, _f32, _int, _vp, _vp],
    "ss_render_backward_finalize": [_vp, _i64, _vp, _i64, _vp, _int, _int, _int, _int, _int, _vp,
                                    _vp, _vp, _vp, _vp, _vp],
    "ss_reference_workspace_bytes": [_i64, _int, _int, _int, _i64, _szp],
    "ss_build_tile_index": [_vp, _vp, _vp, _i64, _int, _int, _int, _int, _f32, _vp, _i64, _vp,
                            _vp, ctypes.c_size_t, _vp, _vp],
    "ss_forward_tiled": [_vp, _vp, _vp, _vp, _vp, _i64, _vp, _i64, _vp, _int, _int, _int, _f32,
                         _int, _int, _f32, _vp, _vp, _vp, ctypes.c_size_t, _vp, _vp],
    "ss_backward_tiled": [_vp, _vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _int,
                          _int, _int, _f32, _int, _int, _f32, _vp, _vp, _vp, _vp, _vp,
                          ctypes.c_size_t, _vp, _vp],
    "ss_batch_project_rs": [_bp, _vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _vp, _vp],
    "ss_batch_tile_index_workspace_bytes": [_bp, _i64, _szp],
    "ss_batch_tile_index_count": [_bp, _vp, _i64, _int, _f32, _vp, _vp, ctypes.c_size_t, _vp,
                                  _vp],
    "ss_batch_tile_index_fill": [_bp, _vp, _i64, _int, _f32, _vp, _vp, _i64, _vp,
                                 ctypes.c_size_t, _vp, _vp],
    "ss_batch_project_rs_index_count": [_bp, _vp, _vp, _vp, _vp, _vp, _i64, _f32, _f32, _int,
                                        _vp, _vp, _vp, ctypes.c_size_t, _vp, ctypes.c_size_t,
                                        _vp, _vp],
    "ss_batch_render_forward": [_bp, _vp, _i64, _vp, _i64, _vp, _int, _f32, _f32, _vp, _vp, _vp,
                                _vp],
    "ss_batch_render_backward": [_bp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _vp, _int, _f32,
                                 _f32, _int, _vp, _vp, _vp, _vp, _int, _vp, ctypes.c_size_t,
                                 _vp, _vp],
    "ss_fit_forward_loss": [_bp, _vp, _i64, _vp, _i64, _vp, _int, _f32, _f32, _vp, _int, _f32,
                            _vp, _vp, _vp, _vp, _vp, _vp],
    "ss_fit_backward_workspace_bytes": [_i64, _i64, _int, _szp],
    "ss_fit_backward": [_bp, _vp, _i64, _vp, _i64, _vp, _f32, _vp, _int, _vp, ctypes.c_size_t,
                        _vp, _vp],
    "ss_ssim_workspace_bytes": [_i64, _szp],
    "ss_ssim_target_stats": [_bp, _vp, _vp, _vp, ctypes.c_size_t, _vp],
    "ss_fit_ssim": [_bp, _vp, _vp, _vp, _vp, _int, _f32, _f32, _vp, _vp, _vp, ctypes.c_size_t,
                    _vp],
    "ss_render_forward_backward": [_vp, _i64, _vp, _i64, _vp, _int, _int, _int, _int, _f32, _f32,
                                   _vp, _vp, _vp, _int, _vp, ctypes.c_size_t, _vp, _vp],
    "ss_fit_forward_backward": [_bp, _vp, _i64, _vp, _i64, _vp, _int, _f32, _f32, _vp, _int,
                                _f32, _vp, _vp, _vp, _int, _vp, ctypes.c_size_t, _vp, _vp],
    "ss_fit_adam_update": [_bp, _vp, _i64, _vp, _i64, _vp, _int, _vp, _f32, _pp, _pp, _pp, _dp,
                           _f64, _f64, _f64, _f32, _vp, _vp, _vp],
    "ss_placement_workspace_bytes": [_int, _int, _szp],
    "ss_density_from_energy": [_vp, _int, _int, _f64, _f64, _vp, _vp, _vp, ctypes.c_size_t, _vp],
    "ss_sample_candidates": [_vp, _int, _int, _vp, _i64, _vp, _vp, _vp, ctypes.c_size_t, _vp],
    "ss_place_gaussians": [_vp, _i64, _vp, _vp, _vp, _vp, _int, _int, _int, _f64, _f64, _f64,
                           _i64, _vp, _vp, _vp, _vp, _vp],
    "ss_sspl1_workspace_bytes": [_i64, _szp],
    "ss_sspl1_dequantize": [ctypes.POINTER(SsSspl1Streams), _vp, _vp, _vp, _vp, _vp, _vp,
                            ctypes.c_size_t, _vp],
    "ss_structure_tensor_workspace_bytes": [_int, _int, _int, _szp],
    "ss_structure_tensor": [_vp, _int, _int, _int, _vp, _int, _vp, _int, _int, _int, _f64, _f64,
                            _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_size_t, _vp],
}
_RESTYPES = {"ss_last_error": ctypes.c_char_p, "ss_splat_record_bytes": ctypes.c_size_t}

_LIB = None
_LOCK = threading.Lock()
CALLS: collections.Counter = collections.Counter()  # entry-point call counts (launch accounting)


class NativeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, name: str, code: int, message: str):
        super().__init__(f"{name} failed (status {code}): {message}")
        self.code = code


def lib():
    """Load (once) and return the CUDA library; raises RuntimeError when it is unavailable."""
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LOCK:
        if _LIB is not None:
            return _LIB
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"structsplat_b200 CUDA library not built ({LIB_PATH} missing); run "
                "`python -m structsplat_b200.build` (there is no CPU fallback)")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _LIB = handle
        return _LIB


def call(name: str, *args) -> None:
    """Invoke a status-returning entry point and raise on failure."""
    CALLS[name] += 1
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        msg = lib().ss_last_error().decode("utf-8", "replace")
        if rc == 1:
            raise ValueError(f"{name}: {msg}")
        raise NativeError(name, rc, msg)


def size_query(name: str, *args) -> int:
    out = ctypes.c_size_t(0)
    call(name, *args, ctypes.byref(out))
    return int(out.value)


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)
