"""Compile the reference CUDA codec from its own sources into oracle/_ref/.

Test infrastructure only.  The reference extension (cuda/csrc/encode.cu,
decode.cu and fastvid_cuda.cpp of generative-workflows/fastvid) is compiled
in place from the read-only reference tree -- its sources are not copied --
with torch's extension builder, for sm_100 (the flags of the reference's
cuda/setup.py:20-23 plus the Blackwell arch), under the module name
``fastvid_ref_C`` so it never shadows the product.  The built module runs only
on a GPU; it pins the CPU oracle through the golden fixtures made by
tests/golden/make_golden.py.

Usage: python oracle/build_ref.py [--reference PATH]
The reference checkout is PATH, else $FASTVID_REFERENCE, else the location
this recipe was written for (REFERENCE_CHECKOUT below).
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# where the read-only reference checkout lives on the build machine; the GPU
# hosts never read it (they use the module built into _ref/)
REFERENCE_CHECKOUT = "/root/reference"


def reference_dir() -> Path | None:
    """The reference checkout, if one is present on this machine."""
    path = Path(os.environ.get("FASTVID_REFERENCE", REFERENCE_CHECKOUT))
    return path if (path / "cuda" / "csrc").is_dir() else None


def built() -> Path | None:
    """The built reference module, if any."""
    found = sorted(OUT.glob("fastvid_ref_C*.so")) if OUT.is_dir() else []
    return found[0] if found else None


def build(reference: Path) -> Path:
    csrc = reference / "cuda" / "csrc"
    sources = [csrc / "fastvid_cuda.cpp", csrc / "decode.cu", csrc / "encode.cu"]
    for src in sources:
        if not src.exists():
            raise FileNotFoundError(src)
    OUT.mkdir(parents=True, exist_ok=True)
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    from torch.utils.cpp_extension import load

    load(
        name="fastvid_ref_C",
        sources=[str(s) for s in sources],
        build_directory=str(OUT),
        extra_cflags=["-O3", "-std=c++17"],
        extra_cuda_cflags=["-O3", "--use_fast_math", "-lineinfo", "-std=c++17"],
        verbose=True,
    )
    built = sorted(OUT.glob("fastvid_ref_C*.so"))
    if not built:
        raise RuntimeError("reference build produced no module")
    return built[0]


def main() -> int:
    parser = argparse.ArgumentParser()
    parser.add_argument("--reference", default=None)
    args = parser.parse_args()
    ref = Path(args.reference) if args.reference else reference_dir()
    if ref is None:
        parser.error("no reference checkout found (pass --reference or set FASTVID_REFERENCE)")
    path = build(ref)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
