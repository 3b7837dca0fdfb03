"""Device status words of the C ABI: Newton failures and bounded-wait
timeouts (fdmap_gpu_status) and the count of non-finite field and fault
values (fdmap_gpu_check_finite, FDMAP_ERR_NONFINITE)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from fdmap_github_b200.native import lib

pytestmark = pytest.mark.gpu


def test_clean_run_reports_ok(require_gpu):
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=10))
    g = GpuDomain(h)
    g.run(1, 8)
    n = C.c_longlong(-1)
    assert lib().fdmap_gpu_status(g._g, C.byref(n)) == 0 and n.value == 0
    assert lib().fdmap_gpu_check_finite(g._g, C.byref(n)) == 0 and n.value == 0
    g.close()


def test_nonfinite_values_are_counted(require_gpu):
    """Values planted from the host (no step runs on them afterwards)."""
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=10))
    g = GpuDomain(h)
    g.run(1, 4)
    F, DF = g.get_fields(True, True)
    F[0, 3, 4] = np.nan
    F[2, 7, 9] = np.inf
    F[5, 20, 40] = -np.inf
    g.set_fields(F, DF)
    assert g.nonfinite_count() == 3
    V = g.get_fault(0, "V")
    V[5] = np.nan
    g.set_fault(0, "V", V)
    assert g.nonfinite_count() == 4
    n = C.c_longlong(0)
    assert lib().fdmap_gpu_check_finite(g._g, C.byref(n)) == -3 and n.value == 4
    assert lib().fdmap_gpu_check_finite(g._g, None) == -3
    g.close()
