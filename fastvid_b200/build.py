"""Build libfastvid_b200.so in-tree with nvcc for sm_100a.

The library is the product: CUDA kernels plus the extern "C" boundary
declared in include/fastvid_b200.h.  It links the CUDA runtime statically, so
it carries no dependency on the runtime version torch ships.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libfastvid_b200.so"
SOURCES = ["fvb_api.cu", "fvb_encode.cu", "fvb_decode.cu"]
HEADERS = ["fvb_common.cuh", "fvb_kernels.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-O3",
    "-Xptxas", "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _inputs():
    yield from (CSRC / s for s in SOURCES)
    yield from (CSRC / h for h in HEADERS)
    yield ROOT / "include" / "fastvid_b200.h"
    yield Path(__file__)


def stale() -> bool:
    if not LIB.exists():
        return True
    built = LIB.stat().st_mtime
    return any(p.stat().st_mtime > built for p in _inputs() if p.exists())


def build(force: bool = False, verbose: bool = False, extra_flags=()) -> Path:
    if not force and not stale():
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, *extra_flags, "-shared", "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr:
        print(res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra_flags=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
    print(LIB)
