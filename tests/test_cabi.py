"""The C ABI library loads on a machine without a GPU and exports every entry
point the public headers declare (no compute calls here)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

from fdmap_github_b200 import native

ROOT = Path(__file__).resolve().parent.parent


def declared_functions(header: Path) -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    return re.findall(r"\b(fdmap_\w+)\s*\(", text)


def test_headers_declare_entry_points():
    names = declared_functions(ROOT / "include" / "fdmap_gpu.h") + declared_functions(ROOT / "include" / "fdmap_host.h")
    assert "fdmap_gpu_create" in names and "fdmap_gpu_time_step" in names and "fdmap_host_init" in names
    assert len(set(names)) == len(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(native.LIB_PATH))
    for h in sorted((ROOT / "include").glob("*.h")):
        for name in declared_functions(h):
            assert hasattr(lib, name), f"{name} declared in {h.name} but not exported"


def test_binding_signatures_cover_headers():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        names.update(declared_functions(h))
    assert names <= set(native.SIGNATURES), sorted(names - set(native.SIGNATURES))
    native.lib()  # binds every signature


def test_error_strings():
    L = native.lib()
    assert L.fdmap_gpu_strerror(0) == b"ok"
    assert b"Newton" in L.fdmap_gpu_strerror(-4)


def test_create_without_gpu_fails_cleanly():
    """No device: create must return an error code, never crash."""
    import torch

    if torch.cuda.is_available():
        return
    from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems

    h = init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3))
    try:
        GpuDomain(h)
    except FdmapError as e:
        assert e.code == -2
    else:
        raise AssertionError("GpuDomain succeeded without a GPU")
