"""fdmap_gpu_fault_max_noalloc (static device scratch, no allocation) against
the existing read-back path fdmap_gpu_get_fault, on two calls in a row."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems

pytestmark = pytest.mark.gpu


def test_fault_max_noalloc_matches_get_fault(require_gpu):
    h = init_domain(problems.rupture_sw(nx=81, ny=41, h=0.5, nt=200))
    g = GpuDomain(h)
    for call in range(2):
        g.run(1 + 40 * call, 40 * (call + 1))
        for field in ("V", "S", "N", "D", "DDs", "trup"):
            expect = float(np.max(np.abs(g.get_fault(0, field))))
            got = g.fault_max_noalloc(0, field)
            assert got == pytest.approx(expect, rel=1e-15, abs=0.0), f"call {call}, {field}"
    # a second handle on the same device shares the scratch; calls in sequence are fine
    g2 = GpuDomain(h)
    assert g2.fault_max_noalloc(0, "S") == pytest.approx(float(np.max(np.abs(g2.get_fault(0, "S")))), rel=1e-15)


def test_fault_max_noalloc_rejects_bad_arguments(require_gpu):
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=3))
    g = GpuDomain(h)
    with pytest.raises(FdmapError):
        g.fault_max_noalloc(3, "V")
