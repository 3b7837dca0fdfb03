"""Builds the CPU oracle (test infrastructure only) into oracle/_build/.

liboracle.so is the C++ restatement of FDMAP's time step, compiled with
-ffp-contract=off so that no fused multiply-adds change the reference's
evaluation order.  OpenMP parallelises loops over grid rows only; each node's
arithmetic is identical for any thread count.

libhost_init.so is the host-side restatement of init_domain
(fdmap_github_b200/csrc/host_init.cpp, the fdmap_host_* entry points of
include/fdmap_host.h) compiled on its own by g++, without the CUDA engine, so
that the CPU arm of bench.py (--impl reference) sets up its domain without
loading any library of the GPU package.
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

HOST_LIB = BUILD / "libhost_init.so"
CSRC = HERE.parent / "fdmap_github_b200" / "csrc"
INCLUDE = HERE.parent / "include"
HOST_SRC = [CSRC / "host_init.cpp"]
HOST_DEPS = HOST_SRC + [CSRC / "body_formulas.h", CSRC / "sbp_tables.h", INCLUDE / "fdmap_desc.h",
                        INCLUDE / "fdmap_host.h"]


def _fresh(lib: Path, deps: list[Path]) -> bool:
    return lib.exists() and all(d.stat().st_mtime <= lib.stat().st_mtime for d in deps)


def build_oracle(force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    if force or not _fresh(LIB, DEPS):
        cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
               *[str(s) for s in SRC], "-o", str(LIB) + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(str(LIB) + ".tmp", LIB)
    if force or not _fresh(HOST_LIB, HOST_DEPS):
        cmd = ["g++", "-std=c++17", "-O3", "-fPIC", "-shared", f"-I{INCLUDE}", f"-I{CSRC}",
               *[str(s) for s in HOST_SRC], "-o", str(HOST_LIB) + ".tmp"]
        subprocess.run(cmd, check=True)
        os.replace(str(HOST_LIB) + ".tmp", HOST_LIB)
    return LIB


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
