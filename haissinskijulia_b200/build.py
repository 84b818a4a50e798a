"""Build the sm_100a tracking library libhaissinski_gpu.so in-tree.

nvcc cross-compiles for sm_100a without a GPU, so this runs on any machine
with the CUDA toolkit.  The shared object lands next to this file, where
``haissinskijulia_b200._lib`` loads it from.

    python -m haissinskijulia_b200.build            # build if sources changed
    python -m haissinskijulia_b200.build --force    # rebuild
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libhaissinski_gpu.so"

CU_SOURCES = ["hj_track.cu", "hj_wake.cu", "hj_api.cu", "hj_batch.cu", "hj_extra.cu",
              "hj_noalloc.cu"]
CPP_SOURCES = ["hj_host.cpp"]
HEADERS = ["hj_device.cuh", "hj_internal.h", "hj_host.h", "hj_launch.h", "hj_ranges.h", "hj_state.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-fno-fast-math"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build the library")
    return cand


def _inputs() -> list[Path]:
    files = [CSRC / f for f in CU_SOURCES + CPP_SOURCES + HEADERS]
    files.append(INCLUDE / "haissinski_gpu.h")
    files.append(Path(__file__))
    return files


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in _inputs())


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compile every CUDA/C++ source for sm_100a and link the shared library."""
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    for src in CU_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, f"-I{INCLUDE}", "-c", str(CSRC / src), "-o", str(obj)]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        _run(cmd, verbose or ptxas_verbose)
        objs.append(obj)
    cxx = os.environ.get("CXX", "g++")
    for src in CPP_SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        _run([cxx, *CXX_FLAGS, f"-I{INCLUDE}", "-I/usr/local/cuda/include", "-c",
              str(CSRC / src), "-o", str(obj)], verbose)
        objs.append(obj)
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
          "-lrt", "-lpthread", "-ldl"], verbose)
    os.replace(tmp, LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v register/smem usage")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, ptxas_verbose=a.ptxas))


if __name__ == "__main__":
    main()
