"""GPU engine vs CPU oracle on identical FDMAP inputs (C ABI through ctypes)."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from oracle.binding import OracleDomain
from tests.parity import assert_fault_close, assert_fields_close, field_errors, rel_err

pytestmark = pytest.mark.gpu


def _pair(text, base=None):
    h = init_domain(text, base)
    return h, GpuDomain(h), OracleDomain(h)


def test_stage_rates_mode3(require_gpu):
    """One stage of rates (interior, 4 side closures, 4 corners, SAT) in mode III."""
    h, g, o = _pair(problems.antiplane_pulse(n=41, L=4.0, nt=2))
    # final step: stage-1 rates only, no update (time_step.f90:133)
    g.time_step_LS(h.t0, h.dt, final_step=True)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    _, DFg = g.get_fields(False, True)
    _, DFo = o.get_fields(False, True)
    assert_fields_close(DFg, DFo, rtol=1e-12, what="DF")


def test_stage_rates_mode2_with_fault(require_gpu):
    h, g, o = _pair(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=2))
    g.time_step_LS(h.t0, h.dt, final_step=True)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    _, DFg = g.get_fields(False, True)
    _, DFo = o.get_fields(False, True)
    assert_fields_close(DFg, DFo, rtol=1e-12, what="DF")
    for b in range(2):
        for s in range(4):
            e = rel_err(g.get_fhat(b, s), o.get_fhat(b, s))
            assert e <= 1e-12, f"Fhat block {b} side {s}: {e}"


def test_antiplane_pulse_full(require_gpu):
    """Config c1 at full size: 201x201, SBP4, absorbing SAT, LS-RK4 CFL 0.5, 500 steps."""
    h, g, o = _pair(problems.antiplane_pulse())
    g.run(1, h.nt)
    o.run(1, h.nt)
    Fg, DFg = g.get_fields(True, True)
    Fo, DFo = o.get_fields(True, True)
    assert_fields_close(Fg, Fo)
    assert_fields_close(DFg, DFo, what="DF")


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_antiplane_operators(require_gpu, fd):
    h, g, o = _pair(problems.antiplane_pulse(n=61, L=6.0, nt=41, fd=fd))
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])


def test_rupture_sw_reduced(require_gpu):
    """Config c2 physics on a coarser grid: two blocks, slip-weakening fault."""
    h, g, o = _pair(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=201))
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
    errs = assert_fault_close(g, o, dt=h.dt, fields=("V", "S", "N", "D", "Ds", "W"))
    assert o.get_fault(0, "D").max() > 1.0  # the rupture did propagate
    print(errs)


@pytest.mark.parametrize("rk", [1, 2, 3, 4])
def test_rk_orders(require_gpu, rk):
    h, g, o = _pair(problems.rupture_sw(nx=81, ny=41, h=0.5, nt=31, rk=rk))
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
    assert_fault_close(g, o, dt=h.dt)
