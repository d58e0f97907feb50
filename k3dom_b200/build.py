"""Build the native library libk3dom_b200.so in-tree for sm_100a.

    python -m k3dom_b200.build [--force] [--verbose]

The shared library is written to k3dom_b200/_lib/ (git-ignored) so it travels with the
source tree. Objects are cached in k3dom_b200/_build/ and rebuilt when a source or header
is newer.
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
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
OBJ_DIR = PKG / "_build"
LIB = OUT_DIR / "libk3dom_b200.so"
INCLUDE = PKG.parent / "include"

CUDA_SOURCES = ["sort.cu", "onesweep.cu", "exactscan.cu", "particles.cu", "cells.cu", "evidence.cu", "dom.cu", "noalloc.cu", "calib.cu"]
CXX_SOURCES = ["params.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--extended-lambda"] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build k3dom_b200")


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "k3dom_b200.h"]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src] + _headers())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> Path:
    nvcc = nvcc_path()
    OUT_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)
    jobs = []
    objs = []
    for s in CUDA_SOURCES:
        src, obj = CSRC / s, OBJ_DIR / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append([nvcc, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)])
    for s in CXX_SOURCES:
        src, obj = CSRC / s, OBJ_DIR / (s + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            jobs.append(["g++", *CXX_FLAGS, "-c", str(src), "-o", str(obj)])
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(lambda c: _run(c, verbose), jobs))
    if force or jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([nvcc, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-cudart", "static"], verbose)
        os.replace(tmp, LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
