"""Access to the reference package installed (unmodified) under ``baseline/_ref`` and to its
CUDA extension built from its own sources for sm_100a (``baseline/build_ref_cuda.py``).

Both travel with the repository snapshot to the GPU host; tests that need them skip when they
are absent.
"""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

BASELINE = Path(__file__).resolve().parent.parent / "baseline"
_EXT_MODULE = None


def _builder():
    if str(BASELINE) not in sys.path:
        sys.path.insert(0, str(BASELINE))
    import build_ref_cuda
    return build_ref_cuda


def reference_modules():
    """(cuda_render, render) of the installed reference package."""
    b = _builder()
    if not b.reference_available():
        pytest.skip("reference package not installed under baseline/_ref")
    if str(b.REF_ROOT) not in sys.path:
        sys.path.insert(0, str(b.REF_ROOT))
    from structsplat import cuda_render, render
    return cuda_render, render


def reference_extension():
    """The reference's own compiled extension module (loaded once per process)."""
    global _EXT_MODULE
    cuda_render, _ = reference_modules()
    if _EXT_MODULE is None:
        b = _builder()
        if b.built_extension_path() is None:
            pytest.skip("reference CUDA extension not built (baseline/build_ref_cuda.py)")
        saved = cuda_render._EXT
        b.load_reference_extension()
        _EXT_MODULE = cuda_render._EXT
        cuda_render._EXT = saved
    return _EXT_MODULE


class installed_extension:
    """Context manager: the reference's ``cuda_render._EXT`` is ``ext`` inside the block."""

    def __init__(self, ext):
        self.ext = ext
        self.cuda_render, _ = reference_modules()

    def __enter__(self):
        self.saved = self.cuda_render._EXT
        self.cuda_render._EXT = self.ext
        return self.cuda_render

    def __exit__(self, *exc):
        self.cuda_render._EXT = self.saved
