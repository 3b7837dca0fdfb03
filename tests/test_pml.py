"""Perfectly matched layer (pml_list; rates_interior_mode2_pml /
rates_boundary_mode2_pml, rates.f90:2024-2619): known answers of the oracle's
restatement, then the GPU against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems
from tests.parity import assert_fields_close


def _oracle(text, steps):
    from oracle.binding import OracleDomain

    h = init_domain(text)
    o = OracleDomain(h)
    o.run(1, steps, nt=1 << 30)
    return h, o


def _strip_pml(text: str) -> str:
    return text.split("&pml_list")[0]


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_undamped_layer_matches_ordinary_rates(fd):
    """With sigma = kappa = 0 the auxiliary fields stay zero and the PML's
    Cartesian rates equal the split-form rates on a uniform grid (to rounding)."""
    text = problems.pml_pulse(n=61, L=6.0, fd=fd, sigma=0.0, bc="absorbing")
    _, o1 = _oracle(text, 30)
    _, o0 = _oracle(_strip_pml(text), 30)
    F1, F0 = o1.get_fields()[0], o0.get_fields()[0]
    assert np.abs(F1 - F0).max() <= 1e-12 * np.abs(F0).max()
    assert not np.any(o1.get_pml("Wx")) and not np.any(o1.get_pml("Wy"))


def test_layer_absorbs_reflections():
    """Free (reflecting) sides: without damping the waves stay in the box;
    the layer takes out all but a fraction of a percent of the kinetic energy
    left in the inner region once the waves have crossed it twice."""
    n, L, w = 81, 8.0, 1.5
    x = np.linspace(0.0, L, n)
    inner = (x >= w) & (x <= L - w)
    ke = []
    for sigma in (None, 0.0):
        _, o = _oracle(problems.pml_pulse(n=n, L=L, width=w, bc="free", sigma=sigma), 300)
        F = o.get_fields()[0]
        ke.append(float((F[0] ** 2 + F[1] ** 2)[np.ix_(inner, inner)].sum()))
    assert ke[0] < 0.01 * ke[1], ke


def test_layer_profile_only_acts_outside_the_inner_region():
    """n > 0: damping sigma*d^n vanishes inside [mx, px] (x) and [my, py] (y)
    and kappa = 0, so Wx stays exactly zero on the columns of the inner region
    and Wy on its rows, while both grow in the layer."""
    n, L, w = 81, 8.0, 2.5
    h, o = _oracle(problems.pml_pulse(n=n, L=L, width=w, bc="absorbing"), 30)
    x, y = h.array("x")[0], h.array("y")[0]  # the grid's own coordinates (rounding included)
    Wx, Wy = o.get_pml("Wx"), o.get_pml("Wy")
    inx = (x >= w) & (x <= L - w)
    iny = (y >= w) & (y <= L - w)
    assert not np.any(Wx[:, inx]) and np.any(Wx[:, ~inx])
    assert not np.any(Wy[:, iny]) and np.any(Wy[:, ~iny])


def test_mode3_ignores_the_layer():
    """set_rates applies the PML branch in mode II only (time_step.f90:354)."""
    text = problems.pml_pulse(n=41, L=4.0, mode=3, width=1.0)
    _, o1 = _oracle(text, 20)
    _, o0 = _oracle(_strip_pml(text), 20)
    assert np.array_equal(o1.get_fields()[0], o0.get_fields()[0])


def test_dissipation_takes_precedence():
    """A block with Cdiss > 0 runs set_rates_dissipation (time_step.f90:242)."""
    text = problems.pml_pulse(n=41, L=4.0, width=1.0, cdiss=0.2)
    _, o1 = _oracle(text, 20)
    _, o0 = _oracle(_strip_pml(text), 20)
    assert np.array_equal(o1.get_fields()[0], o0.get_fields()[0])
    assert not np.any(o1.get_pml("Wx"))


def test_heterogeneous_layer_accepted(tmp_path):
    """A layer in a heterogeneous block runs the homogeneous PML rates with the
    block material (time_step.f90:354-420); tests/test_heterogeneous_variants.py
    checks the arithmetic."""
    text = problems.heterogeneous_ricker(tmp_path, n=31, h=0.1, nt=5)
    text = text.replace("mode=3", "mode=2") + "&pml_list pmlx=T /\n"
    h = init_domain(text, tmp_path)
    assert h.block_pml(0)["pmlx"]


# ---------------------------------------------------------------- GPU

CASES = [
    dict(fd="SBP4"),
    dict(fd="SBP2", kappa=0.7),
    dict(fd="SBP6", npow=3.0),
    dict(fd="SBP4", pmly=False, npow=0.0, sigma=4.0),
    dict(fd="SBP4", pmlx=False, kappa=0.3),
    dict(fd="SBP4", bc="absorbing", width=0.8),
]


@pytest.mark.gpu
@pytest.mark.parametrize("k", range(len(CASES)))
def test_gpu_pml_vs_oracle(require_gpu, k):
    from oracle.binding import OracleDomain

    kw = dict(n=61, L=6.0, width=1.5, bc="free")
    kw.update(CASES[k])
    h = init_domain(problems.pml_pulse(**kw))
    g = GpuDomain(h)
    o = OracleDomain(h)
    steps = 40
    g.run(1, steps, nt=1 << 30)
    o.run(1, steps, nt=1 << 30)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
    for w in ("Wx", "Wy"):
        Wg, Wo = g.get_pml(w), o.get_pml(w)
        scale = max(np.abs(Wo).max(), 1e-300)
        assert np.abs(Wg - Wo).max() <= 1e-10 * scale, f"{CASES[k]}: {w}"
        if (w == "Wx" and kw.get("pmlx", True)) or (w == "Wy" and kw.get("pmly", True)):
            assert np.abs(Wo).max() > 0, "the layer should have been reached"
    g.close()


@pytest.mark.gpu
def test_gpu_pml_state_round_trip(require_gpu):
    """get_pml / set_pml restore the auxiliary fields (checkpoint/resume)."""
    h = init_domain(problems.pml_pulse(n=61, L=6.0, width=1.5))
    g = GpuDomain(h)
    g.run(1, 20, nt=1 << 30)
    F, DF = g.get_fields(True, True)
    W = {w: g.get_pml(w) for w in ("Wx", "Wy")}
    g.run(21, 30, nt=1 << 30)
    ref = g.get_fields()[0]
    g2 = GpuDomain(h)
    g2.set_fields(F, DF)
    for w in W:
        g2.set_pml(w, W[w])
    g2.run(21, 30, nt=1 << 30)
    assert np.array_equal(g2.get_fields()[0], ref)
    g.close()
    g2.close()
