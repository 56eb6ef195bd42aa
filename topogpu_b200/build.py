"""Build ``libtopo_b200.so`` in-tree with nvcc for sm_100a.

Usage: ``python -m topogpu_b200.build`` (or ``__graft_entry__.build()``).
Each translation unit is compiled in parallel, then linked into one shared
library next to this file. The CUDA runtime is linked statically so the
library loads on any box with a driver, without a toolkit.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libtopo_b200.so"
OUT_DBG = PKG / "libtopo_b200_dbg.so"  # -DTOPO_DEBUG_BOUNDS: kernels range-check their gather/scatter indices
SOURCES = ["level0.cu", "kmatvec_xs.cu", "kmatvec_cc.cu", "coarse.cu", "coarsest.cu", "vec.cu", "design.cu", "blockops.cu", "ctx.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-diag-suppress", "177"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libtopo_b200.so")


def sources() -> list[Path]:
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def _stale(out: Path = OUT) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "topo_b200.h", Path(__file__)]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False, debug_bounds: bool = False) -> Path:
    """Compile (if needed) and return the path of the shared library
    (debug_bounds: the range-checked variant libtopo_b200_dbg.so)."""
    out = OUT_DBG if debug_bounds else OUT
    if not force and not _stale(out):
        return out
    nvcc = _nvcc()
    objdir = PKG / ("_build_dbg" if debug_bounds else "_build")
    objdir.mkdir(exist_ok=True)
    extra = ["-DTOPO_DEBUG_BOUNDS"] if debug_bounds else []

    def compile_one(src: Path) -> Path:
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print(r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    p = build(force="--force" in sys.argv, verbose="-v" in sys.argv, debug_bounds="--debug-bounds" in sys.argv)
    print(p)
