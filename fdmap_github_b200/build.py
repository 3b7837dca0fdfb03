"""Builds the native libraries in-tree.

libfdmap_gpu.so   CUDA engine (sm_100a) + host-side domain initialisation,
                  the C ABI of include/fdmap_gpu.h and include/fdmap_host.h.

The shared object is written next to this file so that it travels with the
source tree; it is rebuilt when any source or header is newer than it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libfdmap_gpu.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


# sources whose device arithmetic must round exactly like the host restatement
NO_FMA = {"body_init.cu"}


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))


def _deps() -> list[Path]:
    return _sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, obj: Path, verbose: bool) -> None:
    cmd = [
        NVCC, "-std=c++17", "-O3", *ARCH, "-lineinfo",
        f"-I{INCLUDE}", f"-I{CSRC}",
        "-Xcompiler", "-fPIC,-O3", "-c", str(src), "-o", str(obj),
    ]
    if src.name in NO_FMA:
        cmd.insert(3, "-fmad=false")
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compile libfdmap_gpu.so for sm_100a (cross-compiles without a GPU).

    Each source is compiled to its own object in parallel (objects under
    csrc/_build), then nvcc links the shared object."""
    if not force and not _stale(LIB, _deps()):
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    objdir = CSRC / "_build"
    objdir.mkdir(exist_ok=True)
    srcs = _sources()
    objs = [objdir / (s.name + ".o") for s in srcs]
    with ThreadPoolExecutor(max_workers=max(1, min(len(srcs), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda so: _compile(so[0], so[1], verbose), zip(srcs, objs)))
    cmd = [NVCC, *ARCH, "-shared", *[str(o) for o in objs], "-o", str(LIB) + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
