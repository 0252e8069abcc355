"""Compile the reference's CUDA extension from its sources into oracle/_ref/.

TEST INFRASTRUCTURE ONLY.  Builds cuGAL's pybind11 module ``cuda_kernels``
(``cuda_kernels/kernels.cpp`` + the ``.cu`` files listed in
``cuda_kernels/setup.py:8-16``) with the reference's own nvcc flags
(``-O3 --use_fast_math``, ``cuda_kernels/setup.py:19``) for sm_100, using
torch's extension loader with an explicit source list and an out-of-tree build
directory.  Nothing is written under the reference tree; the output
``oracle/_ref/cuda_kernels*.so`` is git-ignored (a build product, copied with
the working tree to the machine that runs the GPU tests), where
``oracle/ref_gpu.py`` loads it to time and cross-check the reference's FP32 GPU
path.

    python oracle/build_ref.py [--reference <cuGAL checkout>]
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def default_reference() -> str:
    """``CUGAL_REFERENCE``, else a checkout named ``reference`` beside this repository."""
    return os.environ.get("CUGAL_REFERENCE") or str(HERE.parent.parent / "reference")


def build(reference: str | None = None, verbose: bool = False) -> Path | None:
    src = Path(reference or default_reference()) / "cuda_kernels"
    if not src.exists():
        return None
    os.environ.setdefault("TORCH_CUDA_ARCH_LIST", "10.0")
    from torch.utils.cpp_extension import load
    OUT.mkdir(parents=True, exist_ok=True)
    sources = [str(src / f) for f in ["kernels.cpp", "feature_extraction.cu", "adjacency.cu", "sinkhorn_log.cu",
                                      "distance.cu", "regularize.cu", "update_quasi_permutation.cu",
                                      "hungarian/hungarian.cu"]]
    load(name="cuda_kernels", sources=sources, build_directory=str(OUT), extra_cuda_cflags=["-O3", "--use_fast_math"],
         verbose=verbose, is_python_module=True)
    libs = sorted(OUT.glob("cuda_kernels*.so"))
    return libs[0] if libs else None


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=default_reference())
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    out = build(a.reference, a.verbose)
    print(out if out else "reference sources not found; nothing built", file=sys.stderr if out is None else sys.stdout)
