"""Pins for the CPU oracle: answers that follow from FDMAP's own definitions.

The reference ships no tests or golden vectors and cannot be built here
(Fortran + MPI), so the oracle is checked against properties the discrete
scheme must have:
  * the SBP rates are exact for polynomials up to the closure order,
  * the SBP-SAT energy (energy.f90:35-96) does not grow with absorbing or
    free/rigid boundaries,
  * a symmetric rupture set-up stays symmetric,
  * every rate-and-state Newton solve meets the reference's residual
    tolerance atolR = 1e4*eps (friction.f90:931),
  * absorbing boundaries let a pulse leave the domain.
"""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import init_domain, problems
from oracle.binding import OracleDomain

HL = {  # fd_coeff.f90:95, 126, 183-184
    "SBP2": [0.5],
    "SBP4": [0.354166666666667, 1.229166666666667, 0.895833333333333, 1.020833333333333],
    "SBP6": [0.315949074074074, 1.390393518518518, 0.627546296296296, 1.240509259259259, 0.911689814814815,
             1.013912037037037],
}


def hnorm(n, fd):
    H = np.ones(n)
    w = HL[fd]
    H[: len(w)] = w
    H[n - len(w):] = w[::-1]
    return H


def energy_mode3(h, F, rho=2.67, G=2.67 * 3.464 ** 2, fd="SBP4"):
    J = h.array("J")[0]
    Hx, Hy = hnorm(h.nx, fd), hnorm(h.ny, fd)
    e = 0.5 * J * (rho * F[0] ** 2 + (F[1] ** 2 + F[2] ** 2) / G)
    return float(np.sum(e * Hy[:, None] * Hx[None, :]))


@pytest.mark.parametrize("fd,deg", [("SBP2", 1), ("SBP4", 2), ("SBP6", 3)])
def test_rates_exact_for_polynomials(fd, deg):
    """d(sxz)/dx and d(syz)/dy of degree-`deg` polynomials are exact at every
    node away from the SAT-penalised edges (closure order p = deg)."""
    n, L = 31, 3.0
    h = init_domain(problems.antiplane_pulse(n=n, L=L, nt=2, fd=fd, amp=0.0))
    x, y = h.array("x")[0], h.array("y")[0]
    F = h.array("F")
    F[0] = 0.0
    F[1] = (x - 0.7) ** deg          # sxz
    F[2] = 0.5 * (y + 0.3) ** deg    # syz
    o = OracleDomain(h)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    _, DF = o.get_fields(False, True)
    rho = 2.67
    exact = (deg * (x - 0.7) ** (deg - 1) + 0.5 * deg * (y + 0.3) ** (deg - 1)) / rho
    inner = (slice(1, -1), slice(1, -1))
    assert np.max(np.abs(DF[0][inner] - exact[inner])) < 1e-9 * max(1.0, np.abs(exact).max())
    assert np.max(np.abs(DF[1][inner])) < 1e-9 and np.max(np.abs(DF[2][inner])) < 1e-9


@pytest.mark.parametrize("bc", ["absorbing", "free", "rigid"])
def test_energy_does_not_grow(bc):
    h = init_domain(problems.antiplane_pulse(n=61, L=6.0, nt=301, sigma=0.6).replace("'absorbing'", f"'{bc}'"))
    o = OracleDomain(h)
    E = [energy_mode3(h, o.get_fields()[0])]
    for n in range(1, 301):
        o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
        if n % 10 == 0:
            E.append(energy_mode3(h, o.get_fields()[0]))
    E = np.array(E)
    assert np.all(np.diff(E) <= 1e-10 * E[0]), np.diff(E).max() / E[0]
    if bc == "absorbing":
        assert E[-1] < 0.05 * E[0]  # the pulse has left through the absorbing SAT
    else:
        assert E[-1] > 0.99 * E[0]  # free / rigid boundaries conserve energy to the RK dissipation


def test_rupture_symmetry():
    """Uniform prestress, nucleation centred at x = 0: slip is even in x."""
    h = init_domain(problems.rupture_sw(nx=81, ny=41, h=0.5, nt=121))
    o = OracleDomain(h)
    o.run(1, h.nt)
    for f in ("V", "D", "S"):
        v = o.get_fault(0, f)
        assert np.max(np.abs(v - v[::-1])) <= 1e-9 * max(1.0, np.abs(v).max()), f
    assert o.get_fault(0, "D").max() > 0.1


def test_rate_state_newton_residual(tmp_path):
    """After each solve the slip velocity satisfies S = Slock - eta*V and
    S = a*N*asinh(V/(2V0) exp(Psi/a)) to the reference's atolR."""
    text = problems.rough_fault_rs(tmp_path, nx=61, ny=31, h=0.5, nt=40)
    h = init_domain(text, tmp_path)
    o = OracleDomain(h)
    for n in range(1, 30):
        o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt, final_step=(n == 29))
    V, S, N, Psi = (o.get_fault(0, f) for f in ("V", "S", "N", "Psi"))
    a, V0 = 0.01, 1e-6
    Sf = a * N * np.arcsinh(0.5 / V0 * np.exp(Psi / a) * V)
    # the final-step solve used the Psi now stored (no update after it)
    assert np.max(np.abs(Sf - S)) <= 2.3e-12 * 10 + 1e-12 * np.abs(S).max()
    assert o.newton_failures() == 0


def test_locked_interface_energy():
    """Two mode III blocks coupled by a locked interface (interfaces.f90:676-712)
    with rigid outer boundaries: the summed SBP energy is conserved up to the
    RK damping, so the interface SAT coupling neither creates nor loses energy."""
    text = """&problem_list name='locked', nt=201, CFL=0.5d0, RKorder=4 /
&domain_list mode=3, FDmethod='SBP4', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list nx=41, ny=21, LB=0d0,-2d0, LT=0d0,0d0, RB=4d0,-2d0, RT=4d0,0d0 /
&boundaries_list bcL='rigid', bcR='rigid', bcB='rigid', bcT='none' /
&material_list rho=2.67d0, cs=3.464d0 /
&fields_list P5%shape='gaussian', P5%x0=2d0, P5%y0=-0.8d0, P5%Lx=0.3d0, P5%Ly=0.3d0, P5%vz=1d0 /
!---BLOCK2---
&grid_list nx=41, ny=21, LB=0d0,0d0, LT=0d0,2d0, RB=4d0,0d0, RT=4d0,2d0 /
&boundaries_list bcL='rigid', bcR='rigid', bcB='none', bcT='rigid' /
&material_list rho=2.67d0, cs=3.464d0 /
"""
    h = init_domain(text)
    o = OracleDomain(h)
    J = h.array("J")[0]
    Hx = hnorm(41, "SBP4")
    Hy = np.concatenate([hnorm(21, "SBP4"), hnorm(21, "SBP4")])
    G = 2.67 * 3.464 ** 2

    def E(F):
        e = 0.5 * J * (2.67 * F[0] ** 2 + (F[1] ** 2 + F[2] ** 2) / G)
        return float(np.sum(e * Hy[:, None] * Hx[None, :]))

    E0 = E(o.get_fields()[0])
    Es = []
    for n in range(1, h.nt):
        o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
        Es.append(E(o.get_fields()[0]))
    Es = np.array(Es)
    assert np.all(Es <= E0 * (1 + 1e-10))
    assert Es[-1] > 0.98 * E0
    F = o.get_fields()[0]
    assert np.abs(F[0][21:]).max() > 0.05  # the pulse crossed into block 2


def _stage_rates(text, F):
    h = init_domain(text)
    h.array("F")[:] = F
    o = OracleDomain(h)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    return h, o.get_fields(False, True)[1]


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_dissipation_annihilates_constants_and_interior_linears(fd):
    """The artificial dissipation (AI interior / AL closure rows, J-weighted,
    rates.f90:939-1394) vanishes on constant fields everywhere and on linear
    fields away from the closures: the rates with and without it agree."""
    n, L, cd = 41, 4.0, 0.5
    base = problems.antiplane_pulse(n=n, L=L, nt=2, fd=fd, amp=0.0)
    h0 = init_domain(base)
    x, y = h0.array("x")[0], h0.array("y")[0]
    scale = h0.CFL / h0.dt * cd
    for F in (np.stack([np.full_like(x, 0.3), np.full_like(x, 0.2), np.full_like(x, -0.1)]),
              np.stack([0.1 * x + 0.2 * y, 0.3 * x - 0.1 * y, -0.2 * x + 0.05 * y])):
        _, DF0 = _stage_rates(base, F)
        h1, DF1 = _stage_rates(problems.antiplane_pulse(n=n, L=L, nt=2, fd=fd, amp=0.0, cdiss=cd), F)
        assert h1.block_cdiss(0) == pytest.approx(scale)
        nb = {"SBP2": 2, "SBP4": 6, "SBP6": 9}[fd]
        region = (slice(None), slice(None), slice(None)) if np.ptp(F[0]) == 0 else \
            (slice(None), slice(nb, -nb), slice(nb, -nb))
        d = np.abs(DF1 - DF0)[region].max()
        assert d <= 1e-12 * scale * (1 + np.abs(F).max() * L), (fd, d)


def test_dissipation_removes_energy():
    """With energy-conserving free boundaries the dissipative run loses energy
    monotonically, and more than the run without dissipation."""
    def run(cd):
        h = init_domain(problems.antiplane_pulse(n=61, L=6.0, nt=201, sigma=0.3, cdiss=cd).replace("'absorbing'", "'free'"))
        o = OracleDomain(h)
        E = [energy_mode3(h, o.get_fields()[0])]
        for n in range(1, 201):
            o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
            if n % 20 == 0:
                E.append(energy_mode3(h, o.get_fields()[0]))
        return np.array(E)
    E0, E1 = run(0.0), run(0.5)
    assert np.all(np.diff(E1) <= 1e-12 * E1[0])
    assert E1[-1] < E0[-1] * (1 - 1e-4), (E1[-1] / E0[-1])
