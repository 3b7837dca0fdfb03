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


def test_bounded_wait_times_out_and_reports(require_gpu):
    """A wait on an mbarrier that nothing completes (the same bounded-wait
    helper the TMA pipelines use) gives up after its limit and reports
    FDMAP_ERR_TIMEOUT; the context stays usable and the status clears."""
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=10))
    g = GpuDomain(h)
    assert g.status() == 0
    check = lib().fdmap_gpu_test_wait_timeout(g._g, 0.05)
    assert check == 0
    assert g.status() == -5
    g.clear_status()
    assert g.status() == 0
    g.run(1, 4)
    assert g.status() == 0 and g.nonfinite_count() == 0
    g.close()


def _rs_problem():
    from tests.test_parity_matrix import fault_text

    return init_domain(fault_text(law="RSL"))


def test_newton_limit_one_fails_every_solve_like_the_oracle(require_gpu):
    """imax = 1 (fault injection from the host): every rate-and-state solve
    fails and so does its retry -- the reference would stop
    (friction.f90:1014).  The GPU reports FDMAP_ERR_NEWTON_NOCONV with the same
    counts of first failures and failed retries as the oracle."""
    from oracle.binding import OracleDomain

    h = _rs_problem()
    g, o = GpuDomain(h), OracleDomain(h)
    g.set_newton_limit(1)
    o.set_newton_limit(1)
    g.run(1, 3)
    o.run(1, 3)
    gc, oc = g.newton_counts(), o.newton_counts()
    assert oc[0] > 0 and oc[1] == oc[0]
    assert gc == oc
    assert g.status() == -4
    g.close()


def test_newton_retry_from_failed_iterate_matches_oracle(require_gpu):
    """imax = 4: some first attempts fail (about 1400 of the 4100 solves of 20
    steps on the oracle) and are retried from the failed iterate
    (friction.f90:789-790).  GPU and oracle see retries, the retries
    converge on both, and the fields and fault agree as in a normal run."""
    from oracle.binding import OracleDomain

    from tests.parity import assert_fault_close, assert_fields_close

    h = _rs_problem()
    g, o = GpuDomain(h), OracleDomain(h)
    g.set_newton_limit(4)
    o.set_newton_limit(4)
    g.run(1, 20)
    o.run(1, 20)
    gc, oc = g.newton_counts(), o.newton_counts()
    assert oc[0] > 0, "the limit should make some first attempts fail"
    assert abs(gc[0] - oc[0]) <= max(2, oc[0] // 100), (gc, oc)
    assert gc[1] == oc[1] == 0, "every retry should converge"
    assert g.status() == 0
    assert_fields_close(g.get_fields()[0], o.get_fields()[0], what="retry")
    assert_fault_close(g, o, dt=h.dt)
    g.close()
