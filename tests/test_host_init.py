"""Host-side initialisation (init_domain restatement) against known answers."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, init_domain, problems


def test_cartesian_block_metrics():
    h = init_domain(problems.antiplane_pulse(n=41, L=4.0, nt=11))
    assert (h.mode, h.nF, h.nx, h.ny, h.nblocks, h.nifaces) == (3, 3, 41, 41, 1, 0)
    xq, xr, yq, yr, J, Ji = (h.array(n)[0] for n in ("xq", "xr", "yq", "yr", "J", "Ji"))
    assert np.allclose(xq, 0.1, rtol=0, atol=1e-13) and np.allclose(yr, 0.1, rtol=0, atol=1e-13)
    assert np.abs(xr).max() < 1e-13 and np.abs(yq).max() < 1e-13
    assert np.allclose(J * Ji, 1.0, rtol=1e-15)
    x, y = h.array("x")[0], h.array("y")[0]
    assert np.allclose(x[0, :], np.linspace(0, 4, 41), atol=1e-14)
    assert np.allclose(y[:, 0], np.linspace(0, 4, 41), atol=1e-14)


def test_dt_from_cfl():
    """set_dt (domain.f90:1462-1535): dt = CFL*hmin/sqrt(cs^2+cp^2), cp = sqrt(3)*cs."""
    h = init_domain(problems.antiplane_pulse(n=41, L=4.0, nt=11, cfl=0.5))
    c = np.sqrt(3.464 ** 2 + 3 * 3.464 ** 2)
    assert abs(h.dt - 0.5 * h.hmin / c) < 1e-16
    assert abs(h.hmin - 0.1) < 1e-12
    assert h.nt == 11 and h.rk_order == 4


def test_gaussian_pulse_initial_condition():
    h = init_domain(problems.antiplane_pulse(n=41, L=4.0, nt=11, sigma=0.5))
    F = h.array("F")
    x, y = h.array("x")[0], h.array("y")[0]
    r2 = ((x - 2.0) / 0.5) ** 2 + ((y - 2.0) / 0.5) ** 2
    assert np.allclose(F[0], np.exp(-0.5 * r2), rtol=0, atol=1e-15)
    assert np.all(F[1:] == 0.0)


def test_two_block_interface_geometry():
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=3))
    assert (h.nx, h.ny, h.nblocks, h.nifaces) == (41, 42, 2, 1)
    assert h.block_limits(0) == (1, 41, 1, 21) and h.block_limits(1) == (1, 41, 22, 42)
    assert h.iface_n(0) == 41
    F = h.array("F")
    assert np.all(F[4] == -110.0) and np.all(F[3] == 65.0)  # syy0, sxy0 (mode II order vx vy sxx sxy syy szz)
    y = h.array("y")[0]
    assert np.allclose(y[20, :], 0.0) and np.allclose(y[21, :], 0.0)  # both sides of the fault at y = 0


def test_namelist_forms():
    """Positional derived types, %-components, comments, logicals, d-exponents."""
    text = """&problem_list name='t', nt=5, CFL=0.25d0, RKorder=3 / ! comment
&domain_list mode=3, FDmethod='SBP4', nblocks_x=1, nblocks_y=1, exact_metric=F /
!---BLOCK1---
&grid_list nx=21, ny=11, LB%x=0d0, LB%y=0d0, LT=0d0, 1d0, RB = 2.0D0 0.0, RT=2d0,1d0 / trailing
&boundaries_list bcL='free', bcR="rigid", bcB='absorbing', bcT='absorbing' /
&material_list rho=2d0, cs=2d0 /
&fields_list vz0 = 1.5, P1 = 'boxcar', 1d0, 0.5d0, 0.3d0, 0.3d0, 0d0, 0d0, 2d0 /
"""
    h = init_domain(text)
    assert (h.nx, h.ny, h.nt, h.rk_order) == (21, 11, 5, 3)
    x, y = h.array("x")[0], h.array("y")[0]
    assert abs(x[0, -1] - 2.0) < 1e-14 and abs(y[-1, 0] - 1.0) < 1e-14
    F = h.array("F")
    # cs = sqrt(G/rho) = 2 -> cp = 2*sqrt(3); dt from CFL 0.25 and hmin 0.1
    assert abs(h.dt - 0.25 * 0.1 / np.sqrt(4 + 12)) < 1e-12
    inside = ((x - 1.0) / 0.3) ** 2 + ((y - 0.5) / 0.3) ** 2 < 1 - 1e-12
    assert np.allclose(F[0][inside], 1.5 + 2.0) and np.allclose(F[0][~inside & (F[0] != 2.5)], 1.5)


def test_rejects_unsupported_features():
    bad = problems.antiplane_pulse(n=21, L=2.0, nt=3).replace("&fields_list", "&fields_list prestress_from_file=T,")
    with pytest.raises(FdmapError) as e:
        init_domain(bad)
    assert e.value.code == -6
    with pytest.raises(FdmapError):
        init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3).replace("absorbing", "bogus", 1))
    h = init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3).replace(
        "&domain_list mode=3", "&domain_list mode=3, displacement=T, peak=T, energy_balance=T"))
    assert h.displacement and h.peak and h.energy_balance


def test_missing_block_marker():
    text = problems.antiplane_pulse(n=21, L=2.0, nt=3).replace("!---BLOCK1---", "")
    with pytest.raises(FdmapError, match="BLOCK1"):
        init_domain(text)


def test_rough_fault_files(tmp_path):
    text = problems.rough_fault_rs(tmp_path, nx=81, ny=41, h=0.5, nt=3)
    h = init_domain(text, tmp_path)
    y = h.array("y")[0]
    # both blocks share the fault curve: top row of block 1 == bottom row of block 2
    # (up to the rounding of the two transfinite interpolations)
    assert np.allclose(y[40, :], y[41, :], rtol=0, atol=1e-13)
    assert np.abs(y[40, :]).max() > 0
    J = h.array("J")[0]
    assert np.all(J > 0)


def test_dissipation_coefficient_scaled_by_cfl_over_dt():
    """operator_list Cdiss is read per block and scaled by CFL/dt after set_dt
    (domain.f90:172-180, 317-320)."""
    h = init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3, cdiss=0.3))
    assert h.block_cdiss(0) == pytest.approx(0.3 * h.CFL / h.dt, rel=1e-15)
    h2 = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=3, cdiss=0.2))
    assert h2.block_cdiss(0) == h2.block_cdiss(1) == pytest.approx(0.2 * h2.CFL / h2.dt, rel=1e-15)
    assert init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3)).block_cdiss(0) == 0.0
