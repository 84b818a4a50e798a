"""Build the CPU oracle (test infrastructure) into oracle/_build/liboracle.so.

The oracle is compiled without floating-point contraction so that every
rounding of the restatement happens where the reference source places it.
It is portable x86-64 code (no -march=native) because the built object
travels to other machines together with the repository.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "liboracle.so"
SOURCES = [HERE / "oracle.c"]
HEADERS = [HERE / "oracle.h", HERE.parent / "include" / "haissinski_gpu.h"]
CFLAGS = ["-O3", "-fPIC", "-shared", "-std=gnu11", "-ffp-contract=off", "-fno-fast-math"]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(f.stat().st_mtime <= t for f in SOURCES + HEADERS + [Path(__file__)])


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    compilers = [c for c in (os.environ.get("CC"), "/usr/bin/gcc", "gcc") if c]
    # Prefer an OpenMP build (the CPU-baseline leg uses all host cores); a
    # compiler without libgomp still yields a correct serial oracle.
    errors = []
    for omp in (["-fopenmp"], []):
        for cc in compilers:
            cmd = [cc, *CFLAGS, *omp, "-o", str(tmp), *map(str, SOURCES), "-lm"]
            if verbose:
                print(" ".join(cmd))
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode == 0:
                os.replace(tmp, LIB)
                return LIB
            errors.append(r.stdout + r.stderr)
    sys.stderr.write("\n".join(errors))
    raise RuntimeError("oracle build failed")


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
