"""Energy balance (domain_list energy_balance = T; energy_block /
energy_interior, energy.f90:9-96): the stage-1 mechanical energy of every
block as an SBP-norm quadrature.  Known answers on the oracle, then the GPU
against it and the Ebody / Eblock outputs."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, GpuEnsemble, init_domain, problems
from fdmap_github_b200.output import configure_outputs


def _energy(text: str, mode: int) -> str:
    return text.replace(f"&domain_list mode={mode}", f"&domain_list mode={mode}, energy_balance=T")


def test_initial_energy_of_a_gaussian_pulse():
    """E = rho/2 * integral vz^2 = rho/2 * pi sigma^2 for vz = exp(-r^2 / (2 sigma^2))."""
    from oracle.binding import OracleDomain

    h = init_domain(_energy(problems.antiplane_pulse(n=81, L=8.0, nt=10, sigma=0.5), 3))
    assert h.energy_balance
    o = OracleDomain(h)
    o.time_step_LS(h.t0, h.dt, True)
    E = o.get_energy()
    assert abs(E[-1] - 0.5 * 2.67 * np.pi * 0.25) < 1e-9 * E[-1] and E[0] == E[-1]


@pytest.mark.parametrize("bc", ["free", "rigid", "absorbing"])
def test_mode3_energy_does_not_grow(bc):
    from oracle.binding import OracleDomain

    h = init_domain(_energy(problems.antiplane_pulse(n=41, L=4.0, nt=100).replace("absorbing", bc), 3))
    o = OracleDomain(h)
    E = []
    for n in range(1, 121):  # 0.87 s: the pulse reaches every side
        o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
        E.append(o.get_energy()[-1])
    E = np.array(E)
    assert E[0] > 0 and np.all(np.diff(E) <= 1e-12 * E[0])
    if bc == "absorbing":
        assert E[-1] < 0.9 * E[0]  # the pulse leaves through the sides


def _hnorm(n, hl):
    H = np.ones(n)
    H[:len(hl)] = hl
    H[n - len(hl):] = hl[::-1]
    return H


def test_mode2_energy_is_the_reference_quadrature():
    """Mode II as energy_block writes it (energy.f90:67-81): v1 = rho/2 on the
    velocities and v2 = G/2, v3 = G/4, v4 = -G/4 lambda/(3 lambda + 2 G) on the
    stresses -- multiplied by G where a strain energy would divide, so this
    quantity is not conserved; it is kept as the reference computes it."""
    from oracle.binding import OracleDomain

    text = problems.pml_pulse(n=41, L=4.0, sigma=0.0, bc="free").split("&pml_list")[0]
    h = init_domain(_energy(text, 2))
    o = OracleDomain(h)
    o.run(1, 7, nt=1 << 30)
    F = o.get_fields()[0]
    o.time_step_LS(h.t0 + 7 * h.dt, h.dt, True)
    rho, cs, cp = 2.67, 3.464, 6.0
    G, M = rho * cs * cs, rho * cp * cp
    lam = M - 2 * G
    v1, v2, v3, v4 = 0.5 * rho, 0.5 * G, 0.25 * G, -0.25 * G * (lam / (3 * lam + 2 * G))
    dens = (v1 * (F[0] ** 2 + F[1] ** 2) + v2 * F[3] ** 2 + v3 * (F[2] ** 2 + F[4] ** 2 + F[5] ** 2)
            + v4 * (F[2] + F[4] + F[5]) ** 2)
    hl = np.array([0.354166666666667, 1.229166666666667, 0.895833333333333, 1.020833333333333])
    W = np.outer(_hnorm(h.ny, hl), _hnorm(h.nx, hl)) * h.array("J")[0]
    assert abs(o.get_energy()[-1] - np.sum(W * dens)) <= 1e-12 * o.get_energy()[-1]


def test_heterogeneous_energy_uses_the_block_constants(tmp_path):
    """In a heterogeneous medium energy_block still weights with the block's
    material_list constants M%rho, M%G (energy.f90:67-90), not the node's."""
    from oracle.binding import OracleDomain

    het = problems.heterogeneous_ricker(tmp_path, n=31, h=0.1, nt=5)
    h = init_domain(_energy(het, 3), tmp_path)
    assert h.heterogeneous and h.energy_balance
    o = OracleDomain(h)
    o.run(1, 3)
    F = o.get_fields()[0]
    o.time_step_LS(h.t0 + 3 * h.dt, h.dt, True)
    # the quadrature of energy_block with the block constants rho = 2.67, G = rho*cs^2
    hl = np.array([0.354166666666667, 1.229166666666667, 0.895833333333333, 1.020833333333333])
    W = np.outer(_hnorm(h.ny, hl), _hnorm(h.nx, hl)) / h.array("Ji")[0]
    rho, cs = 2.67, 3.464
    G = rho * cs * cs
    E = float(np.sum(0.5 * W * (rho * F[0] ** 2 + (F[1] ** 2 + F[2] ** 2) / G)))
    assert abs(o.get_energy()[-1] - E) <= 1e-12 * abs(E)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["rupture", "pulse", "heterogeneous"])
def test_gpu_energy_vs_oracle(require_gpu, case, tmp_path):
    from oracle.binding import OracleDomain

    if case == "rupture":
        h = init_domain(_energy(problems.rupture_sw(nx=61, ny=31, h=0.4, nt=100), 2))
    elif case == "heterogeneous":
        h = init_domain(_energy(problems.heterogeneous_ricker(tmp_path, n=61, h=0.05, nt=100), 3), tmp_path)
    else:
        h = init_domain(_energy(problems.antiplane_pulse(n=61, L=6.0, nt=100), 3))
    g, o = GpuDomain(h), OracleDomain(h)
    assert np.all(g.get_energy() == 1e40)
    g.run(1, 30)
    o.run(1, 30)
    Eg, Eo = g.get_energy(), o.get_energy()
    assert np.abs(Eg - Eo).max() <= 1e-12 * Eo[-1], (Eg, Eo)
    g.close()


@pytest.mark.gpu
def test_energy_outputs(require_gpu, tmp_path):
    text = _energy(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=30), 2) + """
!---begin:output_list---
EB
Ebody
Etot
0d0 1d10 1
EK
Eblock2
Etot E DE
0d0 1d10 2
!---end:output_list---
"""
    h = init_domain(text)
    g = GpuDomain(h)
    configure_outputs(g, h, text, tmp_path / "e", ring_steps=4)
    nsteps = 12
    g.run(1, nsteps, nt=h.nt)
    g.output_close()
    tot = np.fromfile(tmp_path / "e_EB_Etot.dat", dtype=np.float32)
    blk = np.fromfile(tmp_path / "e_EK_Etot.dat", dtype=np.float32)
    assert tot.size == nsteps and blk.size == nsteps // 2
    assert not np.any(np.fromfile(tmp_path / "e_EK_E.dat", dtype=np.float32))
    assert not np.any(np.fromfile(tmp_path / "e_EK_DE.dat", dtype=np.float32))
    p = GpuDomain(h)
    for n in range(1, nsteps + 1):
        t0 = h.t0 + (n - 1) * h.dt
        p.time_step_LS(t0, h.dt, final_step=True)
        E = p.get_energy()
        assert tot[n - 1] == np.float32(E[-1])
        if (n - 1) % 2 == 0:
            assert blk[(n - 1) // 2] == np.float32(E[1])
        p.time_step_LS(t0, h.dt)


@pytest.mark.gpu
def test_ensemble_rejects_energy(require_gpu, tmp_path):
    text = _energy(problems.ensemble_instance(tmp_path, 0, nx=81, ny=41, nt=20), 2)
    with pytest.raises(FdmapError) as e:
        GpuEnsemble([init_domain(text, tmp_path)])
    assert e.value.code == -6
