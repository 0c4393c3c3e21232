"""The C-ABI library loads and exports every symbol the public header declares.

No compute call is made here (no GPU is needed): only calls that fail argument validation
before touching CUDA, and pure host queries.
"""
from __future__ import annotations

import ctypes
import re
import subprocess

import pytest

from conftest import REPO
from structsplat_b200 import _native, build

HEADER = REPO / "include" / "structsplat_b200.h"


@pytest.fixture(scope="module")
def lib():
    if not _native.LIB_PATH.exists():
        build.build()
    return _native.lib()


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[\w\s\*]+?)\b(ss_\w+)\s*\(", text, re.M)))


def test_header_declares_the_bound_symbols():
    assert declared_symbols() == _native.exported_symbols()


def test_library_exports_every_declared_symbol(lib):
    for name in declared_symbols():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\b(ss_\w+)$", out, re.M))
    assert set(declared_symbols()) <= exported


def test_build_targets_sm100a():
    assert build.ARCH_FLAGS == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_host_queries(lib):
    assert lib.ss_version() == 1
    assert lib.ss_splat_record_bytes() == 64


def _status(lib, name, *args):
    rc = getattr(lib, name)(*args)
    return rc, lib.ss_last_error().decode()


def test_argument_validation_without_gpu(lib):
    size = ctypes.c_size_t(0)
    rc, msg = _status(lib, "ss_tile_index_workspace_bytes", 10, 16, 16, 0, ctypes.byref(size))
    assert rc == 1 and "tile_size" in msg
    rc, msg = _status(lib, "ss_tile_index_workspace_bytes", 10, 16, 16, 33, ctypes.byref(size))
    assert rc == 1 and "tile_size^2 <= 1024" in msg
    rc, msg = _status(lib, "ss_render_forward", None, 0, None, 0, None, 8, 8, 8, 1,
                      ctypes.c_float(1e-8), ctypes.c_float(0.0), None, None, None, None)
    assert rc == 4 and "tile_size" in msg
    rc, msg = _status(lib, "ss_render_forward", None, 0, None, 0, None, 8, 8, 16, 1,
                      ctypes.c_float(0.0), ctypes.c_float(0.0), None, None, None, None)
    assert rc == 1 and "normalization_eps" in msg
    rc, msg = _status(lib, "ss_pack_splats", None, None, None, None, None, -1, 4, 4, None, None)
    assert rc == 1 and "negative" in msg
    rc, msg = _status(lib, "ss_project_rs", None, None, None, None, None, 4, ctypes.c_float(-1.0),
                      ctypes.c_float(3.0), 4, 4, None, None, None, None)
    assert rc == 1 and "dilation" in msg
    rc, msg = _status(lib, "ss_structure_tensor", None, 1, 5, 3, None, 0, None, 0, 0, 0,
                      ctypes.c_double(0.02), ctypes.c_double(0.15), None, None, None, None, None,
                      None, None, None, 0, None)
    assert rc == 1 and "central gradients" in msg
    rc, msg = _status(lib, "ss_render_backward_workspace_bytes", 10, 100, 16, 16, 1,
                      ctypes.byref(size))
    # 12-float partials, two key and two order arrays per entry, begin/end per Gaussian (each
    # 256-byte aligned), then the radix sort's scratch (queried from CUB; none without a GPU)
    fixed = 4864 + 4 * 512 + 256
    assert rc == 0 and size.value >= fixed and size.value % 256 == 0
    rc, msg = _status(lib, "ss_render_backward_workspace_bytes", 10, 100, 16, 16, 0,
                      ctypes.byref(size))
    assert rc == 0 and size.value == 10 * 36


def test_empty_problem_needs_no_device(lib):
    """Zero-sized calls return before any CUDA work."""
    rc, _ = _status(lib, "ss_pack_splats", None, None, None, None, None, 0, 4, 4, None, None)
    assert rc == 0
    rc, _ = _status(lib, "ss_render_forward", None, 0, None, 0, None, 0, 7, 16, 1,
                    ctypes.c_float(1e-8), ctypes.c_float(0.0), None, None, None, None)
    assert rc == 0


def test_batch_validation_without_gpu(lib):
    size = ctypes.c_size_t(0)
    rc, msg = _status(lib, "ss_batch_tile_index_workspace_bytes", None, 10, ctypes.byref(size))
    assert rc == 1 and "null batch" in msg
    b = _native.SsBatch(images=0, tile_size=16, tiles=0, pixels=0)
    rc, msg = _status(lib, "ss_batch_tile_index_workspace_bytes", ctypes.byref(b), 10,
                      ctypes.byref(size))
    assert rc == 1 and "at least one image" in msg
    b = _native.SsBatch(images=1, tile_size=16, tiles=4, pixels=16)
    rc, msg = _status(lib, "ss_batch_tile_index_workspace_bytes", ctypes.byref(b), 10,
                      ctypes.byref(size))
    assert rc == 1 and "table pointer" in msg
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size query reads no table
    b = _native.SsBatch(images=1, tile_size=16, tiles=4, pixels=16, image_table=dummy,
                        pixel_base=dummy, gaussian_base=dummy, gaussian_image=dummy,
                        tile_image=dummy)
    rc, _ = _status(lib, "ss_batch_tile_index_workspace_bytes", ctypes.byref(b), 10,
                    ctypes.byref(size))
    assert rc == 0 and size.value > 0
    b.tile_size = 8
    rc, msg = _status(lib, "ss_batch_render_forward", ctypes.byref(b), None, 0, None, 0, None, 1,
                      ctypes.c_float(1e-8), ctypes.c_float(0.0), None, None, None, None)
    assert rc == 4 and "tile_size" in msg
    b.tile_size = 32
    rc, msg = _status(lib, "ss_fit_forward_loss", ctypes.byref(b), None, 0, None, 0, None, 1,
                      ctypes.c_float(1e-8), ctypes.c_float(0.0), None, 7, ctypes.c_float(1e-3),
                      None, None, None, None, None, None)
    assert rc == 1 and "loss_kind" in msg
    rc, msg = _status(lib, "ss_fit_backward_workspace_bytes", 10, 100, 1, ctypes.byref(size))
    # 12-float partials, two key and two order arrays per entry, begin/end per Gaussian (each
    # 256-byte aligned), the radix sort's scratch (queried from CUB; none without a GPU), then
    # the five gradient arrays of the Adam step (each 256-byte aligned)
    fixed = 4864 + 4 * 512 + 256
    grads = 5 * 256
    assert rc == 0 and size.value >= fixed + grads and size.value % 256 == 0
    rc, msg = _status(lib, "ss_fit_backward_workspace_bytes", 10, 100, 0, ctypes.byref(size))
    assert rc == 0 and size.value == 512 + grads  # moments 360 B, then the gradients
    lrs = (ctypes.c_double * 5)(*([1e-2] * 5))
    ptrs = (ctypes.c_void_p * 5)()
    rc, msg = _status(lib, "ss_fit_adam_update", ctypes.byref(b), None, 10, None, 0, None, 0,
                      None, ctypes.c_float(0.0), ptrs, ptrs, ptrs, lrs, 0.9, 0.999, 1e-8,
                      ctypes.c_float(-1.0), None, None, None)
    assert rc == 1 and "null" in msg


def test_backward_warps_knob_validation(lib):
    rc, msg = _status(lib, "ss_set_backward_warps", 8, 4)
    assert rc == 4 and "tile_size" in msg
    rc, msg = _status(lib, "ss_set_backward_warps", 32, 12)
    assert rc == 1 and "0, 8 or 16" in msg
    assert lib.ss_get_backward_warps(16) == 8 and lib.ss_get_backward_warps(32) == 8
    assert lib.ss_set_backward_warps(32, 16) == 0 and lib.ss_get_backward_warps(32) == 16
    assert lib.ss_set_backward_warps(32, 0) == 0 and lib.ss_get_backward_warps(32) == 8
    assert lib.ss_get_backward_warps(7) == -1


def test_forward_chunk_knob_validation(lib):
    rc, msg = _status(lib, "ss_set_forward_chunk", 8, 64)
    assert rc == 4 and "tile_size" in msg
    rc, msg = _status(lib, "ss_set_forward_chunk", 32, 100)
    assert rc == 1 and "0, 64, 128 or 256" in msg
    assert lib.ss_get_forward_chunk(16) == 256 and lib.ss_get_forward_chunk(32) == 256
    assert lib.ss_set_forward_chunk(32, 64) == 0 and lib.ss_get_forward_chunk(32) == 64
    assert lib.ss_set_forward_chunk(32, 0) == 0 and lib.ss_get_forward_chunk(32) == 256
    assert lib.ss_get_forward_chunk(7) == -1


def test_dependent_launch_switch(lib):
    """Programmatic dependent launch is on by default; the switch takes 0 or 1 only."""
    assert lib.ss_get_dependent_launch() == 1
    rc, msg = _status(lib, "ss_set_dependent_launch", 2)
    assert rc == 1 and "0 or 1" in msg
    assert lib.ss_set_dependent_launch(0) == 0 and lib.ss_get_dependent_launch() == 0
    assert lib.ss_set_dependent_launch(1) == 0 and lib.ss_get_dependent_launch() == 1
