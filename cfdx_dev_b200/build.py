"""Build libcfdxg.so in-tree (cfdx_dev_b200/_lib/) for sm_100a.

Usage: python -m cfdx_dev_b200.build [--force]

CUDA sources are compiled by nvcc for sm_100a only.  Translation units whose
FP64 results must match the reference bit for bit are built with
``-fmad=false`` so no multiply-add is contracted into an FMA; host C++ units
use ``-ffp-contract=off`` for the same reason.
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
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
OBJ = OUT / "obj"
INCLUDE = PKG.parent / "include"
LIB = OUT / "libcfdxg.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(INCLUDE), *ARCH]
# units whose FP64 arithmetic is compared bit-exactly with the reference
EXACT_CUDA = {"assembly.cu", "vcycle.cu", "krylov.cu", "matrix.cu", "capi.cu", "galerkin.cu", "gauge.cu"}
CXXFLAGS = ["-O2", "-std=c++17", "-fPIC", "-pthread", "-ffp-contract=off", f"-I{INCLUDE}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, headers: list[Path]) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _compile(src: Path, force: bool, headers: list[Path]) -> Path:
    obj = OBJ / (src.name + ".o")
    if not force and not _stale(src, obj, headers):
        return obj
    if src.suffix == ".cu":
        flags = list(NVCC_COMMON)
        flags += ["-fmad=false"] if src.name in EXACT_CUDA else ["-fmad=true"]
        cmd = [nvcc(), *flags, "-c", str(src), "-o", str(obj)]
    else:
        cmd = [os.environ.get("CXX", "g++"), *CXXFLAGS, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> Path:
    OBJ.mkdir(parents=True, exist_ok=True)
    srcs = sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))
    headers = _headers()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, headers), srcs))
    if force or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcusolver", "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


def main(argv: list[str] | None = None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    build(force=args.force, verbose=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
