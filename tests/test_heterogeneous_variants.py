"""Artificial dissipation and the perfectly matched layer in a heterogeneous
medium.  set_rates_dissipation takes the heterogeneous routines
(rates_h_dissipation_*, rates_heterogeneous.f90:920-1997; time_step.f90:555-751);
set_rates runs the PML rates with the block's homogeneous material before its
heterogeneous branch (time_step.f90:354-420) and keeps the node's nu for szz
(486-490).  Known answers on the oracle (a uniform medium file reproduces the
homogeneous block), then the GPU against the oracle on random media."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from tests.parity import assert_fields_close

HOM = "&material_list rho=2.67d0, cs=3.464d0, cp=6.0d0 /"
HET = "&material_list heterogeneous=T, filename='medium.dat', rho=2.67d0, cs=3.464d0, cp=6.0d0 /"


def _medium(tmp_path, n, seed=None, std=0.08):
    """rho, cs, cp over an n x n grid (i fastest on disk); uniform without a seed."""
    rho = np.full((n, n), 2.67)
    cs = np.full((n, n), 3.464)
    cp = np.full((n, n), 6.0)
    if seed is not None:
        rng = np.random.default_rng(seed)
        x = np.linspace(0, 1, n)
        X, Y = np.meshgrid(x, x, indexing="ij")
        for a in (rho, cs, cp):
            k = rng.uniform(1, 3, 2)
            a *= 1.0 + std * np.sin(2 * np.pi * k[0] * X + rng.uniform(0, 6)) * np.cos(2 * np.pi * k[1] * Y)
    np.concatenate([rho.T.ravel(), cs.T.ravel(), cp.T.ravel()]).tofile(tmp_path / "medium.dat")


def _pml_text(tmp_path, n, het, seed=None, cdiss=0.0):
    text = problems.pml_pulse(n=n, L=(n - 1) * 0.1, width=1.5, bc="free", cdiss=cdiss)
    assert HOM in text
    if het:
        _medium(tmp_path, n, seed)
        text = text.replace(HOM, HET)
    return text


def _diss_text(tmp_path, n, mode, fd="SBP4", cdiss=0.4, seed=None, het=True):
    text = problems.pml_pulse(n=n, L=(n - 1) * 0.1, width=1.5, bc="absorbing", cdiss=cdiss, mode=mode, fd=fd)
    text = text.split("&pml_list")[0]
    if het:
        _medium(tmp_path, n, seed)
        text = text.replace(HOM, HET)
    return text


def _oracle(text, base, steps):
    from oracle.binding import OracleDomain

    h = init_domain(text, base)
    o = OracleDomain(h)
    o.run(1, steps, nt=1 << 30)
    return h, o


def test_uniform_medium_pml_block_is_the_homogeneous_block(tmp_path):
    _, o_het = _oracle(_pml_text(tmp_path, 41, True), tmp_path, 25)
    _, o_hom = _oracle(_pml_text(tmp_path, 41, False), None, 25)
    Fa, Fb = o_het.get_fields()[0], o_hom.get_fields()[0]
    assert np.abs(Fb).max() > 0
    np.testing.assert_allclose(Fa, Fb, rtol=0, atol=1e-13 * np.abs(Fb).max())
    np.testing.assert_allclose(o_het.get_pml("Wx"), o_hom.get_pml("Wx"), rtol=0,
                               atol=1e-13 * np.abs(o_hom.get_pml("Wx")).max())


@pytest.mark.parametrize("mode", [2, 3])
def test_uniform_medium_dissipation_is_the_homogeneous_dissipation(tmp_path, mode):
    _, o_het = _oracle(_diss_text(tmp_path, 41, mode), tmp_path, 25)
    _, o_hom = _oracle(_diss_text(tmp_path, 41, mode, het=False), None, 25)
    Fa, Fb = o_het.get_fields()[0], o_hom.get_fields()[0]
    assert np.abs(Fb).max() > 0
    np.testing.assert_allclose(Fa, Fb, rtol=0, atol=1e-12 * np.abs(Fb).max())


def _sbp4_norm(n):
    """Diagonal SBP4 norm with unit spacing (boundary weights 17/48, 59/48,
    43/48, 49/48, interior 1)."""
    w = np.ones(n)
    hl = [17 / 48, 59 / 48, 43 / 48, 49 / 48]
    w[:4] = hl
    w[-4:] = hl[::-1]
    return w


@pytest.mark.parametrize("cdiss", [0.0, 0.4])
def test_heterogeneous_energy_does_not_grow(tmp_path, cdiss):
    """SBP-SAT energy of a heterogeneous mode III medium with absorbing sides,
    E = 1/2 sum H J (rho vz^2 + (sxz^2 + syz^2)/G), never grows from step to
    step, with or without the dissipative rates."""
    from oracle.binding import OracleDomain

    h = init_domain(_diss_text(tmp_path, 41, 3, cdiss=cdiss, seed=4), tmp_path)
    o = OracleDomain(h)
    rho, G, J = h.array("rho")[0], h.array("G")[0], h.array("J")[0]
    W = np.outer(_sbp4_norm(h.ny), _sbp4_norm(h.nx)) * J
    E = []
    for n in range(1, 61):
        F = o.get_fields()[0]
        E.append(0.5 * np.sum(W * (rho * F[0] ** 2 + (F[1] ** 2 + F[2] ** 2) / G)))
        o.run(n, n, nt=1 << 30)
    E = np.array(E)
    assert E[0] > 0
    assert np.all(np.diff(E) <= 1e-13 * E[0])
    if cdiss > 0:
        # the dissipative rates remove energy the plain rates keep
        h0 = init_domain(_diss_text(tmp_path, 41, 3, cdiss=0.0, seed=4), tmp_path)
        o0 = OracleDomain(h0)
        o0.run(1, 59, nt=1 << 30)
        F0 = o0.get_fields()[0]
        E0 = 0.5 * np.sum(W * (rho * F0[0] ** 2 + (F0[1] ** 2 + F0[2] ** 2) / G))
        assert E[-1] < E0


def test_dissipation_damps_a_heterogeneous_medium(tmp_path):
    """The dissipative rates remove energy that the plain rates keep."""
    _, o_d = _oracle(_diss_text(tmp_path, 41, 3, seed=4, cdiss=0.6), tmp_path, 40)
    _, o_0 = _oracle(_diss_text(tmp_path, 41, 3, seed=4, cdiss=0.0), tmp_path, 40)
    Fd, F0 = o_d.get_fields()[0], o_0.get_fields()[0]
    assert np.sum(Fd[0] ** 2) < np.sum(F0[0] ** 2)


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("mode,fd", [(3, "SBP2"), (3, "SBP4"), (3, "SBP6"), (2, "SBP4"), (2, "SBP6")])
def test_gpu_heterogeneous_dissipation_stage_rates(require_gpu, tmp_path, mode, fd):
    """One stage on random fields: every AI / AL weight, closure row and the
    node material enter."""
    from oracle.binding import OracleDomain

    h = init_domain(_diss_text(tmp_path, 41, mode, fd=fd, seed=7), tmp_path)
    F = h.array("F")
    F[:] = np.random.default_rng(3).standard_normal(F.shape)
    g, o = GpuDomain(h), OracleDomain(h)
    g.time_step_LS(h.t0, h.dt, final_step=True)
    o.time_step_LS(h.t0, h.dt, final_step=True)
    assert_fields_close(g.get_fields(False, True)[1], o.get_fields(False, True)[1], rtol=1e-12, what="DF")
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [2, 3])
def test_gpu_heterogeneous_dissipation_run(require_gpu, tmp_path, mode):
    from oracle.binding import OracleDomain

    h = init_domain(_diss_text(tmp_path, 61, mode, seed=5), tmp_path)
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 60, nt=1 << 30)
    o.run(1, 60, nt=1 << 30)
    Fo = o.get_fields()[0]
    assert np.abs(Fo).max() > 0
    assert_fields_close(g.get_fields()[0], Fo)
    g.close()


@pytest.mark.gpu
def test_gpu_heterogeneous_pml_run(require_gpu, tmp_path):
    from oracle.binding import OracleDomain

    h = init_domain(_pml_text(tmp_path, 61, True, seed=9), tmp_path)
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 60, nt=1 << 30)
    o.run(1, 60, nt=1 << 30)
    Fo = o.get_fields()[0]
    assert np.abs(Fo).max() > 0
    assert_fields_close(g.get_fields()[0], Fo)
    for name in ("Wx", "Wy"):
        a, b = g.get_pml(name), o.get_pml(name)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), name
    g.close()
