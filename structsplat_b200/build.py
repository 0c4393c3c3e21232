"""Build the CUDA library ``structsplat_b200/_lib/libstructsplat_b200.so`` for sm_100a.

Each ``csrc/*.cu`` is compiled by nvcc (in parallel) to an object and linked into one shared
library with the CUDA runtime linked statically, so the library loads in any process with a
CUDA driver.  Objects are rebuilt only when a source or header is newer.

    python -m structsplat_b200.build [-v] [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
OBJ_DIR = PKG / "_lib" / "obj"
LIB_PATH = PKG / "_lib" / "libstructsplat_b200.so"
HEADERS = [REPO / "include" / "structsplat_b200.h", *sorted(CSRC.glob("*.cuh"))]

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists() and shutil.which(cand) is None:
        raise RuntimeError("nvcc not found; set NVCC or put CUDA's bin directory on PATH")
    return cand


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=()) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    if not sources:
        raise RuntimeError(f"no CUDA sources under {CSRC}")
    compiler = nvcc()
    jobs = []
    for src in sources:
        obj = OBJ_DIR / (src.stem + ".o")
        if force or _stale(obj, [src, *HEADERS]):
            cmd = [compiler, *ARCH_FLAGS, *NVCC_FLAGS, *extra_flags, "-I", str(REPO / "include"),
                   "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        if verbose and (res.stdout or res.stderr):
            print(res.stdout + res.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [OBJ_DIR / (s.stem + ".o") for s in sources]
    if force or jobs or _stale(LIB_PATH, objs):
        cmd = [compiler, *ARCH_FLAGS, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB_PATH),
               *map(str, objs), "-cudart", "static"]
        run(cmd)
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
