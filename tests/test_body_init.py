"""On-device initialisation: the host does the O(nx + ny) part of init_domain,
the engine builds the grid, metrics, Jacobian, initial body fields and side
impedances on the device and reduces hmin / hmax for set_dt.  The device body
must equal the host restatement's bit for bit (last-bit exp() differences
allowed in 'smooth' / 'gaussian' perturbations), and the runs that follow
must agree with the host-initialised ones."""
from __future__ import annotations

import math

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, GpuEnsemble, init_domain, problems

SKEWED = """&problem_list name='skew', nt=21, CFL=0.4d0, RKorder=4 /
&domain_list mode=2, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={nx}, ny={ny}, LB=0d0, 0d0, LT=0.3d0, 2d0, RB=3d0, -0.2d0, RT=3.2d0, 2.4d0,
  bndLmap=1.5d0, bndBmap=-2d0 /
&boundaries_list bcL='absorbing', bcR='free', bcB='rigid', bcT='absorbing' /
&material_list rho=2.5d0, cs=3d0, cp=5.5d0 /
&fields_list sxx0=-40d0, syy0=-50d0, sxy0=10d0,
  P1='boxcar', 1.5d0, 1d0, 0.5d0, 0.4d0, 0.3d0, 0d0, 0d0, 0d0, 0d0, 0d0, 0d0, 0d0, 0d0,
  P2%shape='linear', P2%x0=1d0, P2%y0=1d0, P2%Lx=3d0, P2%Ly=2d0, P2%sxy=2d0,
  P3%shape='triangle', P3%x0=2d0, P3%y0=1d0, P3%Lx=0.6d0, P3%Ly=0.6d0, P3%vy=0.2d0,
  P4%shape='smooth', P4%x0=1.2d0, P4%y0=0.8d0, P4%Lx=0.5d0, P4%Ly=0.7d0, P4%syy=-3d0 /
&operator_list Cdiss={cdiss} /
"""


def _skewed(fd="SBP4", nx=61, ny=47, cdiss="0d0"):
    return SKEWED.format(fd=fd, nx=nx, ny=ny, cdiss=cdiss)


def _cases(tmp_path):
    """(name, input text, base dir, exp-based perturbation present)"""
    return [
        ("pulse", problems.antiplane_pulse(n=61, L=6.0, nt=21), None, True),
        ("rupture", problems.rupture_sw(nx=81, ny=41, h=0.1, nt=21), None, False),
        ("rough", problems.rough_fault_rs(tmp_path, nx=81, ny=41, h=0.25, nt=21), tmp_path, False),
        ("het", problems.heterogeneous_ricker(tmp_path, n=41, h=0.1, nt=21, seed=1), tmp_path, False),
        ("skewed4", _skewed(), None, True),
        ("skewed6", _skewed("SBP6", 53, 41), None, True),
        ("skewed2", _skewed("SBP2", 37, 29), None, True),
        ("cdiss", _skewed(cdiss="0.3d0"), None, True),
        # perfectly matched layer: damping profile pow() on the device grid
        ("pml", problems.pml_pulse(n=61, L=6.0, nt=21, width=1.5, bc="free"), None, True),
    ]


# ---------------------------------------------------------------- host side (CPU)

@pytest.mark.parametrize("k", range(9))
def test_deferred_host_init_matches_full(tmp_path, k):
    name, text, base, _ = _cases(tmp_path)[k]
    full = init_domain(text, base)
    dev = init_domain(text, base, body_on_device=True)
    assert (dev.mode, dev.nF, dev.nx, dev.ny, dev.nblocks, dev.nifaces, dev.rk_order) == \
        (full.mode, full.nF, full.nx, full.ny, full.nblocks, full.nifaces, full.rk_order)
    # the O(nx*ny) body is absent on the host; the time step waits for the spacings
    for a in ("F", "DF", "x", "y", "xq", "xr", "yq", "yr", "J", "Ji"):
        with pytest.raises(KeyError):
            dev.array(a)
    assert dev.spacing_pending and math.isnan(dev.dt) and dev.t0 == full.t0
    for b in range(full.nblocks):
        assert dev.block_limits(b) == full.block_limits(b)
        for s in range(4):
            assert np.array_equal(dev.side_array(b, s, "F0"), full.side_array(b, s, "F0"))
            assert np.array_equal(dev.side_array(b, s, "normal"), full.side_array(b, s, "normal"))
            with pytest.raises(KeyError):
                dev.side_array(b, s, "M")
    for i in range(full.nifaces):
        assert dev.iface_info(i) == full.iface_info(i)
        for a, c in zip(dev.iface_xy(i), full.iface_xy(i)):
            assert np.array_equal(a, c)
    # finishing set_dt with the host's spacings reproduces the host's time step exactly
    dev.set_spacing(full.hmin, full.hmax)
    assert not dev.spacing_pending
    assert (dev.dt, dev.CFL, dev.nt, dev.hmin, dev.hmax) == (full.dt, full.CFL, full.nt, full.hmin, full.hmax)
    for b in range(full.nblocks):
        assert dev.block_cdiss(b) == full.block_cdiss(b)


def test_set_spacing_rules():
    text = problems.antiplane_pulse(n=21, L=2.0, nt=3)
    with pytest.raises(FdmapError):
        init_domain(text).set_spacing(0.1, 0.1)  # body already on the host
    dev = init_domain(text, body_on_device=True)
    with pytest.raises(FdmapError):
        dev.set_spacing(0.0, 0.1)
    assert dev.spacing_pending


def test_init_ex_rejects_unknown_flags():
    import ctypes as C

    from fdmap_github_b200.native import lib

    h = C.c_void_p()
    text = problems.antiplane_pulse(n=21, L=2.0, nt=3).encode()
    assert lib().fdmap_host_init_ex(text, None, 6, C.byref(h)) == -1
    assert not h


# ---------------------------------------------------------------- device side

def _assert_fields(a, b, exp_shapes, what):
    if exp_shapes:
        # exp() of the device and of the host may differ in the last bit
        np.testing.assert_allclose(a, b, rtol=4e-16, atol=1e-300, err_msg=what)
    else:
        assert np.array_equal(a, b), what


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(9))
def test_device_body_matches_host_body(require_gpu, tmp_path, k):
    name, text, base, exp_shapes = _cases(tmp_path)[k]
    full = init_domain(text, base)
    dev = init_domain(text, base, body_on_device=True)
    gf = GpuDomain(full)
    gd = GpuDomain(dev)
    t0, dt, CFL, hmin, hmax, nt = gd.time_params()
    assert (hmin, hmax) == (full.hmin, full.hmax), name
    assert (t0, dt, CFL, nt) == (full.t0, full.dt, full.CFL, full.nt), name
    assert (dev.dt, dev.CFL, dev.nt, dev.hmin, dev.hmax) == (full.dt, full.CFL, full.nt, full.hmin, full.hmax)
    metrics = ["xq", "xr", "yq", "yr", "Ji"] + (["J"] if name == "cdiss" else [])
    for m in metrics:
        a, b = gd.get_metric(m), gf.get_metric(m)
        assert np.array_equal(a, b), f"{name}: metric {m}"
        if m != "J":
            assert np.array_equal(b, full.array(m)[0]), f"{name}: uploaded {m}"
    for b in range(full.nblocks):
        for s in range(4):
            Md = gd.get_side_impedance(b, s)
            assert np.array_equal(Md, gf.get_side_impedance(b, s)), f"{name}: impedances of block {b} side {s}"
            assert np.array_equal(Md, full.side_array(b, s, "M")), f"{name}: host impedances of block {b} side {s}"
    Fd, DFd = gd.get_fields(True, True)
    Ff, DFf = gf.get_fields(True, True)
    _assert_fields(Fd, Ff, exp_shapes, f"{name}: initial fields")
    assert np.array_equal(DFd, DFf), f"{name}: initial rates"
    for b in range(full.nblocks):
        for s in range(4):
            _assert_fields(gd.get_fhat(b, s), gf.get_fhat(b, s), exp_shapes, f"{name}: initial hat variables")
    # the runs that follow
    nsteps = 12
    gd.run(1, nsteps)
    gf.run(1, nsteps)
    Fd, _ = gd.get_fields()
    Ff, _ = gf.get_fields()
    if exp_shapes:
        scale = np.abs(Ff).max()
        assert np.abs(Fd - Ff).max() <= 1e-13 * scale, name
    else:
        assert np.array_equal(Fd, Ff), f"{name}: fields after {nsteps} steps"
    if name == "pml":
        for w in ("Wx", "Wy"):
            a, b = gd.get_pml(w), gf.get_pml(w)
            assert np.abs(b).max() > 0 and np.abs(a - b).max() <= 1e-13 * np.abs(b).max(), f"pml {w}"
    for i in range(full.nifaces):
        if full.iface_info(i)[3] == 1:
            for f in ("V", "S", "N", "D", "Psi"):
                assert np.array_equal(gd.get_fault(i, f), gf.get_fault(i, f)), f"{name}: fault {f}"
    gd.close()
    gf.close()


@pytest.mark.gpu
def test_ensemble_with_device_bodies(require_gpu, tmp_path):
    sizes = [(81, 41), (97, 65), (161, 41)]
    texts = [problems.ensemble_instance(tmp_path, seed, nx=nx, ny=ny, nt=41) for seed, (nx, ny) in enumerate(sizes)]
    hosts = [init_domain(t, tmp_path) for t in texts]
    devs = [init_domain(t, tmp_path, body_on_device=True) for t in texts]
    ef, ed = GpuEnsemble(hosts), GpuEnsemble(devs)
    assert [h.dt for h in devs] == [h.dt for h in hosts]
    assert ed.dt == ef.dt
    ef.run(1, 15, dt=ef.dt)
    ed.run(1, 15, dt=ed.dt)
    for k in range(len(sizes)):
        Fe, DFe = ed[k].get_fields(True, True)
        Ff, DFf = ef[k].get_fields(True, True)
        assert np.array_equal(Fe, Ff) and np.array_equal(DFe, DFf), f"instance {k}"
        assert np.array_equal(ed[k].get_fault(0, "V"), ef[k].get_fault(0, "V"))
    ed.close()
    ef.close()
