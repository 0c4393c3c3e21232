"""Build the reference's own CUDA extension, unmodified, for sm_100a.

The reference package is installed (unmodified) into ``baseline/_ref`` with::

    python -m pip install --no-index --no-build-isolation --no-deps \
        --find-links /opt/wheelhouse --target baseline/_ref <copy of the reference>

Its renderer JIT-compiles ``structsplat/cuda/render_ext.{cpp,cu}`` on first use
(``structsplat/cuda_render.py:21-49``), which takes minutes and writes into the user's
cache.  This script performs that same compile ahead of time, with the same sources and
``-O3`` flags plus an explicit sm_100a target, into ``baseline/_ref/ext/`` so the built
module travels with the repository snapshot to the GPU host.  ``load_reference_extension``
then imports the prebuilt module and installs it as the reference's ``_EXT`` so the
reference's public ``render_cuda_exact`` runs its stock code path on it.

This is baseline plumbing only: nothing in ``structsplat_b200`` imports it.
"""
from __future__ import annotations

import importlib.machinery
import importlib.util
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_ROOT = HERE / "_ref"
EXT_DIR = REF_ROOT / "ext"
EXT_NAME = "structsplat_render_ext"


def reference_available() -> bool:
    return (REF_ROOT / "structsplat" / "render.py").is_file()


def built_extension_path() -> Path | None:
    for cand in sorted(EXT_DIR.glob(f"{EXT_NAME}*.so")):
        return cand
    return None


def build(verbose: bool = False) -> Path:
    """Compile the reference extension for sm_100a into baseline/_ref/ext."""
    if not reference_available():
        raise RuntimeError("reference package is not installed under baseline/_ref")
    from torch.utils.cpp_extension import load

    src = REF_ROOT / "structsplat" / "cuda"
    EXT_DIR.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0a")
    load(
        name=EXT_NAME,
        sources=[str(src / "render_ext.cpp"), str(src / "render_ext.cu")],
        extra_cflags=["-O3"],
        extra_cuda_cflags=["-O3", "-gencode", "arch=compute_100a,code=sm_100a"],
        with_cuda=True,
        build_directory=str(EXT_DIR),
        verbose=verbose,
    )
    path = built_extension_path()
    if path is None:
        raise RuntimeError("reference extension build produced no .so")
    return path


def load_reference_extension():
    """Import the prebuilt reference extension and hand it to the reference's wrapper.

    Returns the reference ``cuda_render`` module, whose ``render_cuda_exact`` now runs on the
    prebuilt sm_100a extension.
    """
    path = built_extension_path()
    if path is None:
        raise RuntimeError("reference CUDA extension not built (run baseline/build_ref_cuda.py)")
    import torch  # noqa: F401  (the extension links against torch's libraries)

    if str(REF_ROOT) not in sys.path:
        sys.path.insert(0, str(REF_ROOT))
    loader = importlib.machinery.ExtensionFileLoader(EXT_NAME, str(path))
    spec = importlib.util.spec_from_file_location(EXT_NAME, str(path), loader=loader)
    module = importlib.util.module_from_spec(spec)
    loader.exec_module(module)
    from structsplat import cuda_render

    cuda_render._EXT = module
    return cuda_render


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
