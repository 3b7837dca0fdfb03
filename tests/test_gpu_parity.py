"""GPU engine vs CPU oracle on identical FDMAP inputs (C ABI through ctypes)."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from oracle.binding import OracleDomain
from tests.parity import assert_fault_close, assert_fields_close, assert_law_parity, field_errors, rel_err

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


def test_graph_replay_matches_direct_steps(require_gpu, tmp_path):
    """fdmap_gpu_run replays a captured CUDA graph per step with the step clock
    on the device; it must reproduce per-step fdmap_gpu_time_step bit for bit
    (stage times enter the rupture times and the source amplitude)."""
    for text, base in ((problems.rupture_sw(nx=81, ny=41, h=0.5, nt=40), None),
                       (problems.heterogeneous_ricker(tmp_path, n=61, h=0.05, nt=40), tmp_path)):
        h = init_domain(text, base)
        g1, g2 = GpuDomain(h), GpuDomain(h)
        g1.run(1, h.nt)
        for n in range(1, h.nt + 1):
            g2.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt, final_step=(n == h.nt))
        F1, D1 = g1.get_fields(True, True)
        F2, D2 = g2.get_fields(True, True)
        assert np.array_equal(F1, F2) and np.array_equal(D1, D2)
        if h.nifaces:
            for f in ("V", "S", "D", "trup", "Psi"):
                assert np.array_equal(g1.get_fault(0, f), g2.get_fault(0, f)), f


def test_heterogeneous_point_source(require_gpu, tmp_path):
    """Config c5 physics at reduced size: heterogeneous mode III medium, Ricker
    point force, free top surface."""
    text = problems.heterogeneous_ricker(tmp_path, n=101, h=0.05, nt=121)
    h, g, o = _pair(text, tmp_path)
    g.run(1, h.nt)
    o.run(1, h.nt)
    Fo = o.get_fields()[0]
    assert np.abs(Fo[0]).max() > 0
    assert_fields_close(g.get_fields()[0], Fo)


def test_rough_fault_rate_state(require_gpu, tmp_path):
    """Config c3 physics at reduced size: curvilinear blocks around a rough
    fault, regularised rate-and-state friction with flash heating (RFL)."""
    text = problems.rough_fault_rs(tmp_path, nx=121, ny=61, h=0.25, nt=161)
    h, g, o = _pair(text, tmp_path)
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_law_parity(g, o, "RFL", h, h.nt, dt=h.dt)
    assert g.newton_failures() == 0 and o.newton_failures() == 0


def _random_fields(h, seed):
    rng = np.random.default_rng(seed)
    F = h.array("F")
    F[:] = rng.standard_normal(F.shape)


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_dissipation_stage_rates_mode3(require_gpu, fd):
    """One stage of the dissipative rates (set_rates_dissipation) on a random
    field, so every AI / AL weight and every closure row is exercised."""
    h = init_domain(problems.antiplane_pulse(n=41, L=4.0, nt=2, fd=fd, cdiss=0.4))
    _random_fields(h, 1)
    g, o = GpuDomain(h), OracleDomain(h)
    g.time_step_LS(h.t0, h.dt, final_step=True)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    assert_fields_close(g.get_fields(False, True)[1], o.get_fields(False, True)[1], rtol=1e-12, what="DF")


def test_dissipation_stage_rates_mode2(require_gpu):
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=2, cdiss=0.3))
    _random_fields(h, 2)
    g, o = GpuDomain(h), OracleDomain(h)
    g.time_step_LS(h.t0, h.dt, final_step=True)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    assert_fields_close(g.get_fields(False, True)[1], o.get_fields(False, True)[1], rtol=1e-12, what="DF")


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_dissipation_pulse_run(require_gpu, fd):
    h, g, o = _pair(problems.antiplane_pulse(n=61, L=6.0, nt=61, fd=fd, cdiss=0.5))
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])


def test_dissipation_rupture_run(require_gpu):
    h, g, o = _pair(problems.rupture_sw(nx=121, ny=61, h=0.25, nt=121, cdiss=0.3))
    g.run(1, h.nt)
    o.run(1, h.nt)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
    assert_fault_close(g, o, dt=h.dt, fields=("V", "S", "N", "D"))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [2, 3])
def test_side_displacement_vs_oracle(require_gpu, mode):
    """Boundary displacement of every side (integrated from the hat velocities,
    fields.f90:1083-1276) against the oracle, and the jump across the fault
    equal to the slip register Ds."""
    from oracle.binding import OracleDomain

    if mode == 2:
        h = init_domain(problems.rupture_sw(nx=81, ny=41, h=0.25, nt=200))
    else:
        h = init_domain(problems.antiplane_pulse(n=61, L=6.0, nt=200))
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 40)
    o.run(1, 40)
    sides = [(b, s) for b in range(h.nblocks) for s in range(4)]
    gpu = {k: g.get_side_displacement(*k) for k in sides}
    ora = {k: o.get_side_u(*k) for k in sides}
    # errors relative to the largest displacement (rate) on any side: sides
    # far from the source carry values at the rounding level of that scale
    for q in range(2):
        scale = max(np.abs(ora[k][q]).max() for k in sides)
        assert scale > 0
        for k in sides:
            assert np.abs(gpu[k][q] - ora[k][q]).max() <= 1e-10 * scale, (k, q)
    if mode == 2:
        Um, Up = g.get_side_displacement(0, 3)[0], g.get_side_displacement(1, 2)[0]
        Ds = g.get_fault(0, "Ds")
        assert np.abs(Ds).max() > 0
        assert np.abs((Up[0] - Um[0]) - Ds).max() <= 1e-12 * np.abs(Ds).max()
    g.close()
