"""GPU against the oracle across the configuration space of the time step:
every friction law (friction.f90:700-826, 1147-1264), both interface
directions, the load shapes (friction.f90:1348-1369), forced rupture,
thermal-pressurisation p0, regularised normal stress, rupture on slip, a
rotated fault, and every outer boundary condition (boundaries.f90:155-377),
in mode II and mode III.  Small two-block problems, 30 steps each."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain
from tests.parity import assert_fields_close, assert_law_parity


def _f(x: float) -> str:
    return repr(float(x)).replace("e", "d") if "e" in repr(float(x)) else repr(float(x)) + "d0"


def fault_text(mode=2, law="SW", direction="y", ld="gaussian", bc="absorbing", fd="SBP4", n=41, h=0.25,
               friction_extra="", extra_blocks="", nt=31, coupling="friction") -> str:
    """Two blocks of n x (n//2 + 1) nodes (direction 'y': stacked, fault y = 0;
    'x': side by side, fault x = 0) with a frictional interface, or with
    coupling='locked' a welded interface (locked_interface_mode2/3,
    interfaces.f90:676-772) crossed by a Gaussian velocity pulse that starts
    in block 1 one km from it."""
    m = n // 2 + 1
    L, W = (n - 1) * h, (m - 1) * h
    if direction == "y":
        g1 = f"nx={n}, ny={m}, LB={_f(-L/2)},{_f(-W)}, LT={_f(-L/2)},0d0, RB={_f(L/2)},{_f(-W)}, RT={_f(L/2)},0d0"
        g2 = f"nx={n}, ny={m}, LB={_f(-L/2)},0d0, LT={_f(-L/2)},{_f(W)}, RB={_f(L/2)},0d0, RT={_f(L/2)},{_f(W)}"
        b1 = f"bcL='{bc}', bcR='{bc}', bcB='{bc}', bcT='none'"
        b2 = f"bcL='{bc}', bcR='{bc}', bcB='none', bcT='{bc}'"
        dom = "nblocks_x=1, nblocks_y=2"
        stress = "syy0=-100d0, sxy0=58d0, sxx0=-100d0" if mode == 2 else "syy0=-100d0, syz0=58d0"
    else:
        g1 = f"nx={m}, ny={n}, LB={_f(-W)},{_f(-L/2)}, LT={_f(-W)},{_f(L/2)}, RB=0d0,{_f(-L/2)}, RT=0d0,{_f(L/2)}"
        g2 = f"nx={m}, ny={n}, LB=0d0,{_f(-L/2)}, LT=0d0,{_f(L/2)}, RB={_f(W)},{_f(-L/2)}, RT={_f(W)},{_f(L/2)}"
        b1 = f"bcL='{bc}', bcR='none', bcB='{bc}', bcT='{bc}'"
        b2 = f"bcL='none', bcR='{bc}', bcB='{bc}', bcT='{bc}'"
        dom = "nblocks_x=2, nblocks_y=1"
        # with the normal along +x the fault-tangent direction is -y, so the
        # shear traction on the fault is -sxy
        stress = "sxx0=-100d0, sxy0=-58d0, syy0=-100d0" if mode == 2 else "sxx0=-100d0, sxz0=58d0"
    ldline = f"ld%shape='{ld}', ld%R=1.5d0, ld%S=20d0, ld%x0=0d0, ld%y0=0d0, ld%T=0d0," if ld else ""
    if law == "SW":
        params = "sw%fs=0.68d0, sw%fd=0.52d0, sw%Dc=0.2d0,"
    elif law in ("frictionless", "locked"):
        params = ""
    else:
        params = "rs%a=0.01d0, rs%b=0.014d0, rs%V0=1d-6, rs%f0=0.6d0, rs%L=0.05d0, rs%fw=0.2d0, rs%Vw=0.1d0, Psi0=0.6d0,"
    if coupling == "locked":
        x0, y0 = ("0.5d0", "-1d0") if direction == "y" else ("-1d0", "0.5d0")
        v = "P5%vx=1d0, P5%vy=0.5d0" if mode == 2 else "P5%vz=1d0"
        stress += f", P5%shape='gaussian', P5%x0={x0}, P5%y0={y0}, P5%Lx=0.6d0, P5%Ly=0.6d0, {v}"
    blk = f"&material_list rho=2.67d0, cs=3.464d0, cp=6d0 /\n&fields_list {stress} /\n"
    return f"""&problem_list name='matrix', nt={nt}, CFL=0.5d0, RKorder=4 /
&domain_list mode={mode}, FDmethod='{fd}', {dom} /
!---BLOCK1---
&grid_list {g1} /
&boundaries_list {b1} /
{blk}!---BLOCK2---
&grid_list {g2} /
&boundaries_list {b2} /
{blk}{extra_blocks}!---IFACE1---
&interface_list coupling='{coupling}', direction='{direction}' /
""" + ("" if coupling == "locked" else f"""&friction_list friction_law='{law}', {params} {ldline}
  rup_field='V', rup_threshold=1d-3 {friction_extra} /
""")


CASES = {
    # friction laws, mode II, fault y = 0
    "SW": dict(),
    "SL": dict(law="SL"),
    "FL": dict(law="FL"),
    "RSL": dict(law="RSL"),
    "RFL": dict(law="RFL"),
    "RSF": dict(law="RSF"),
    "RAL": dict(law="RAL"),
    "frictionless": dict(law="frictionless", ld=""),
    # mode III
    "III-SW": dict(mode=3),
    "III-RAL": dict(mode=3, law="RAL"),
    "III-x-RSL": dict(mode=3, law="RSL", direction="x"),
    # fault x = 0
    "x-SW": dict(direction="x", ld="boxcar"),
    "x-RFL": dict(direction="x", law="RFL"),
    # load shapes
    "ld-uniform": dict(ld="uniform"),
    "ld-linear": dict(ld="linear"),
    "ld-smooth_boxcar": dict(ld="smooth_boxcar"),
    "ld-triangle": dict(ld="triangle"),
    "ld-smooth": dict(ld="smooth"),
    "ld-ramp": dict(ld="boxcar", friction_extra=", ld%T=0.1d0"),
    # forced rupture, thermal pressurisation p0, regularised N, rupture on slip, rotated fault
    "forced": dict(mode=3, ld="", friction_extra=", force=T, kn%fd=0.52d0, kn%dfdx=0.2d0, kn%vL=-2d0, kn%vR=2d0, "
                                               "kn%xL=0.2d0, kn%xR=-0.2d0, kn%tmax=4d0"),
    "tp-p0": dict(law="RSL", extra_blocks="", friction_extra=" /\n&thermpres_list n=64, p0=10d0"),
    "reg": dict(law="RSL", friction_extra=", reg=T"),
    "rup-D": dict(friction_extra=", rup_field='D'"),
    "angle": dict(friction_extra=", angle=10d0"),
    "lock-window": dict(friction_extra=", xlockm=-2d0, xlockp=2d0, flock=0.8d0"),
    # outer boundary conditions
    "bc-free": dict(bc="free"),
    "bc-rigid": dict(bc="rigid"),
    "bc-absorbing-0": dict(bc="absorbing-0"),
    "bc-free-0": dict(bc="free-0"),
    "bc-rigid-0": dict(bc="rigid-0"),
    "bc-absorbing-velocity": dict(bc="absorbing-velocity"),
    "bc-free-velocity": dict(bc="free-velocity"),
    "III-bc-free": dict(mode=3, bc="free"),
    "III-bc-rigid": dict(mode=3, bc="rigid"),
    # operators
    "SBP2": dict(fd="SBP2"),
    "SBP6": dict(fd="SBP6", n=49),
}


def test_every_case_initialises_and_runs_on_the_oracle():
    from oracle.binding import OracleDomain

    for name, kw in CASES.items():
        h = init_domain(fault_text(**kw))
        o = OracleDomain(h)
        o.run(1, 3)
        F = o.get_fields()[0]
        assert np.all(np.isfinite(F)), name


# welded interfaces in both modes and both directions (interfaces.f90:676-772)
LOCKED = {
    "locked-II-y": dict(coupling="locked"),
    "locked-II-x": dict(coupling="locked", direction="x"),
    "locked-III-y": dict(coupling="locked", mode=3),
    "locked-III-x": dict(coupling="locked", mode=3, direction="x"),
}


def test_locked_cases_initialise_and_run_on_the_oracle():
    from oracle.binding import OracleDomain

    for name, kw in LOCKED.items():
        h = init_domain(fault_text(**kw))
        assert h.iface_info(0)[3] == 0, name  # FDMAP_COUPLING_LOCKED
        o = OracleDomain(h)
        o.run(1, 3)
        assert np.all(np.isfinite(o.get_fields()[0])), name


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(LOCKED))
def test_locked_gpu_vs_oracle(require_gpu, name):
    """The pulse crosses the welded interface: fields and the hat variables of
    both interface sides against the oracle."""
    from oracle.binding import OracleDomain

    from tests.parity import rel_err

    h = init_domain(fault_text(**LOCKED[name]))
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 30)
    o.run(1, 30)
    Fo = o.get_fields()[0]
    assert_fields_close(g.get_fields()[0], Fo, what=name)
    sides = ((0, 3), (1, 2)) if LOCKED[name].get("direction", "y") == "y" else ((0, 1), (1, 0))
    for b, sd in sides:
        e = rel_err(g.get_fhat(b, sd), o.get_fhat(b, sd))
        assert e <= 1e-10, f"{name}: hat variables of block {b} side {sd}: {e}"
    # the pulse reached block 2 through the interface
    n_half = h.ny // 2 if LOCKED[name].get("direction", "y") == "y" else None
    v2 = Fo[0, n_half:, :] if n_half else Fo[0, :, h.nx // 2:]
    assert np.abs(v2).max() > 1e-3
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_vs_oracle(require_gpu, name):
    from oracle.binding import OracleDomain

    h = init_domain(fault_text(**CASES[name]))
    g, o = GpuDomain(h), OracleDomain(h)
    steps = 30
    g.run(1, steps)
    o.run(1, steps)
    law = CASES[name].get("law", "SW")
    assert_law_parity(g, o, law, h, steps, dt=h.dt, what=name)
    assert g.newton_failures() == o.newton_failures() == 0
    assert np.abs(o.get_fault(0, "V")).max() > 1e-3, f"{name}: the fault should slip"
    g.close()


# 200 steps of every law whose Newton solves all converge there (the
# log-strength law 'FL' fails its retries on this rupture after ~100 steps,
# where the reference would stop, friction.f90:1014)
LONG = ["SW", "SL", "RSL", "RFL", "RSF", "RAL", "III-RAL", "x-RFL", "lock-window"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", LONG)
def test_gpu_vs_oracle_200_steps(require_gpu, name):
    """Longer runs: the rate-and-state laws are held to the spread of the
    reference's own answer within its Newton tolerance (tests/parity.py),
    the explicit laws to 1e-10."""
    from oracle.binding import OracleDomain

    h = init_domain(fault_text(**CASES[name], nt=201))
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 200)
    o.run(1, 200)
    law = CASES[name].get("law", "SW")
    assert_law_parity(g, o, law, h, 200, dt=h.dt, what=name)
    assert g.newton_counts() == o.newton_counts()
    g.close()
