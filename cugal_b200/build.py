"""Build the sm_100a kernel library ``cugal_b200/lib/libfugal_b200.so`` in-tree.

    python -m cugal_b200.build [--verbose-ptxas]

Every ``csrc/*.cu`` is compiled by nvcc for ``sm_100a`` (in parallel), then
linked into one shared library with the C ABI declared in
``include/fugal_b200.h``.  Rebuilds only what changed (by mtime, headers
included).  No GPU is needed to build.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = ROOT / "_build" / "obj"
LIB_DIR = PKG / "lib"
LIB = LIB_DIR / "libfugal_b200.so"
HEADERS = [ROOT / "include" / "fugal_b200.h", *CSRC.glob("*.cuh"), *CSRC.glob("*.h")]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fvisibility=hidden", "-DFUGAL_BUILDING_LIBRARY"]


def nvcc() -> str:
    for cand in [os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"]:
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose_ptxas: bool = False, force: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB_DIR.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []

    def compile_one(src: Path) -> tuple[Path, str]:
        obj = OBJ / (src.stem + ".o")
        if force or verbose_ptxas or _stale(obj, [src, *HEADERS]):
            cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
            return obj, r.stderr
        return obj, ""

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, sources))
    if verbose_ptxas:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    if force or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose-ptxas", action="store_true")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(args.verbose_ptxas, args.force))
