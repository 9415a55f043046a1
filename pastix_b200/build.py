"""Build the in-tree shared library ``pastix_b200/lib/libpastix_b200.so``.

All CUDA sources are compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``); the host analysis is plain C++.
Objects go to ``pastix_b200/_build`` and are rebuilt when their source or a
header is newer.  Usage: ``python -m pastix_b200.build [-v] [-j N]``.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libpastix_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I", str(ROOT / "include")] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-I", str(ROOT / "include")]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home() -> Path:
    return Path(nvcc_path()).resolve().parent.parent


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.hpp")) + sorted((ROOT / "include").glob("*.h"))


def _stale(src: Path, obj: Path, deps: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *deps])


def _compile(src: Path, verbose: bool, extra: list[str]) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(src, obj, _headers()):
        return obj
    if src.suffix == ".cu":
        cmd = [nvcc_path(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{r.stdout}\n{r.stderr}")
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj


def build(verbose: bool = False, jobs: int | None = None, ptxas_verbose: bool = False) -> Path:
    """Compile every source and link the shared library; returns its path."""
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose, extra), srcs))
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc_path(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs),
               "-L", str(cuda_home() / "lib64"), "-lcudart", "-Xlinker", f"-rpath={cuda_home() / 'lib64'}"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--ptxas", action="store_true", help="print register / smem usage")
    a = ap.parse_args()
    print(build(a.verbose, a.jobs, a.ptxas))
    return 0


if __name__ == "__main__":
    sys.exit(main())
