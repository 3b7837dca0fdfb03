"""Builds the CPU oracle (test infrastructure only) into oracle/_build/.

liboracle.so is the C++ restatement of FDMAP's time step, compiled with
-ffp-contract=off so that no fused multiply-adds change the reference's
evaluation order.  OpenMP parallelises loops over grid rows only; each node's
arithmetic is identical for any thread count.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
LIB = BUILD / "liboracle.so"
SRC = [HERE / "fdmap_oracle.cpp"]
DEPS = SRC + [HERE / "fdmap_oracle.h", HERE.parent / "include" / "fdmap_desc.h"]


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if not force and LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in DEPS):
        return LIB
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
           *[str(s) for s in SRC], "-o", str(LIB) + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
