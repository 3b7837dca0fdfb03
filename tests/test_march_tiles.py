"""Tile shapes of the interior march kernel (strip width x rows per row
group), the single-domain autotuner, and the march's extras variant
(dissipation, PML, forcing, body displacement and peak motion, heterogeneous
mode II), which replaces the tiled interior kernel for those domains.

Per-node arithmetic does not depend on the tile shape, so every shape gives
the same bits; the extras variant is checked against the tiled kernel
(FDMAP_STENCIL=tile) and against the oracle."""
from __future__ import annotations

import os

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems
from tests.parity import assert_fields_close

pytestmark = pytest.mark.gpu


def _tiled(h):
    os.environ["FDMAP_STENCIL"] = "tile"
    try:
        return GpuDomain(h)
    finally:
        del os.environ["FDMAP_STENCIL"]


def test_every_tile_gives_the_same_bits(require_gpu):
    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=60))
    ref = None
    for tile in (0, 1, 2, 3):
        g = GpuDomain(h)
        g.set_tile(tile)
        assert g.tile()[0] == tile
        g.run(1, 40)
        F, DF = g.get_fields(True, True)
        V = g.get_fault(0, "V")
        if ref is None:
            ref = (F, DF, V)
        else:
            assert np.array_equal(F, ref[0]) and np.array_equal(DF, ref[1]) and np.array_equal(V, ref[2]), tile
        g.close()


def test_tile_refused_where_the_stencil_is_wider(require_gpu):
    """SBP6 (half-width 3) cannot march in row groups of 2 rows."""
    h = init_domain(problems.antiplane_pulse(n=61, L=6.0, nt=5, fd="SBP6"))
    g = GpuDomain(h)
    with pytest.raises(FdmapError) as e:
        g.set_tile(1)
    assert e.value.code == -6
    assert g.tile()[0] == 0  # unchanged
    g.run(1, 3)


def test_tuner_picks_a_tile_and_leaves_the_state(require_gpu):
    h = init_domain(problems.rupture_sw(nx=321, ny=161, h=0.125, nt=100))
    g, ref = GpuDomain(h), GpuDomain(h)
    g.run(1, 10)
    ref.run(1, 10)
    tile, ms = g.tune(steps=3)
    assert tile in (0, 1, 2, 3) and ms > 0 and g.tile()[0] == tile
    g.run(11, 30)
    ref.run(11, 30)
    assert np.array_equal(g.get_fields()[0], ref.get_fields()[0])
    assert np.array_equal(g.get_fault(0, "V"), ref.get_fault(0, "V"))


def _het_pml(t, cdiss=0.0, mode=2):
    from tests.test_heterogeneous_variants import _diss_text, _pml_text

    return _pml_text(t, 61, True, seed=3) if cdiss == 0.0 else _diss_text(t, 61, mode, cdiss=cdiss, seed=4)


def _extras(text: str, mode: int) -> str:
    return text.replace(f"&domain_list mode={mode}", f"&domain_list mode={mode}, displacement=T, peak=T")


CASES = {
    "dissipation-II": lambda t: problems.rupture_sw(nx=81, ny=41, h=0.5, nt=60, cdiss=0.3),
    "dissipation-III": lambda t: problems.antiplane_pulse(n=61, L=6.0, nt=60, cdiss=0.2),
    "pml-II": lambda t: problems.pml_pulse(n=81, L=8.0, width=2.0, nt=60),
    "forcing-III": lambda t: problems.gaussian_forcing(n=61, L=60.0, nt=40),
    "extras-II": lambda t: _extras(problems.rupture_sw(nx=81, ny=41, h=0.5, nt=60), 2),
    "het-pml-II": lambda t: _het_pml(t),
    "het-dissipation-II": lambda t: _het_pml(t, cdiss=0.4),
    "het-dissipation-III": lambda t: _het_pml(t, cdiss=0.4, mode=3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_march_extras_against_tiled_kernel_and_oracle(require_gpu, tmp_path, name):
    from oracle.binding import OracleDomain

    text = CASES[name](tmp_path)
    h = init_domain(text, tmp_path)
    g, t = GpuDomain(h), _tiled(h)
    assert g.tile()[0] in (0, 1, 2, 3)  # the march serves it
    with pytest.raises(FdmapError):
        t.tile()  # the tiled kernel
    g.run(1, 30)
    t.run(1, 30)
    o = OracleDomain(h)
    o.run(1, 30)
    Fg, Ft, Fo = g.get_fields()[0], t.get_fields()[0], o.get_fields()[0]
    assert_fields_close(Fg, Fo, what=f"{name} march")
    assert_fields_close(Fg, Ft, rtol=1e-13, what=f"{name} march vs tiled")
    if h.pml_fields() != (False, False):
        for w in ("Wx", "Wy"):
            assert_fields_close(g.get_pml(w), o.get_pml(w), what=f"{name} {w}")
    if h.displacement:
        for a, b, what in zip(g.get_displacement() + g.get_peak(), o.get_displacement() + o.get_peak(),
                              ("U", "DU", "pgv", "pga")):
            err = float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)
            assert err <= 1e-10, f"{name} {what}: {err}"


def test_heterogeneous_mode2_marches_in_thin_row_groups(require_gpu, tmp_path):
    """The heterogeneous mode II rings do not fit with 4-row groups; the
    engine takes the 2-row shape and matches the oracle."""
    from oracle.binding import OracleDomain

    from tests.test_heterogeneous_variants import _medium

    _medium(tmp_path, 61, seed=7)
    text = problems.pml_pulse(n=61, L=6.0, width=1.5, bc="absorbing").split("&pml_list")[0].replace(
        "&material_list rho=2.67d0, cs=3.464d0, cp=6.0d0 /",
        "&material_list heterogeneous=T, filename='medium.dat', rho=2.67d0, cs=3.464d0, cp=6.0d0 /")
    h = init_domain(text, tmp_path)
    assert h.heterogeneous and h.mode == 2
    g = GpuDomain(h)
    assert g.tile()[2] == 2
    g.run(1, 40)
    o = OracleDomain(h)
    o.run(1, 40)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
