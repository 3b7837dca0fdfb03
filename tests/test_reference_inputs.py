"""The reference's own example inputs (problems/*.in and gp229/*.in of the
FDMAP source tree) through the host initialisation and the oracle, where that
tree is given (FDMAP_SOURCE_TREE; skipped when unset).  The binary side
files their MATLAB scripts write (kali_input.m, pointsource_heterogeneous.m,
LLWgaussianForcing.m) are generated here from the formulas those scripts use."""
from __future__ import annotations

import os
import re
from pathlib import Path

import numpy as np
import pytest

from fdmap_github_b200 import init_domain, problems

_TREE_ENV = os.environ.get("FDMAP_SOURCE_TREE")
TREE = Path(_TREE_ENV) if _TREE_ENV else None
pytestmark = pytest.mark.skipif(TREE is None or not (TREE / "problems").is_dir(),
                                reason="FDMAP source tree not given (FDMAP_SOURCE_TREE)")


def _text(rel: str) -> str:
    return (TREE / rel).read_text()


def _oracle_steps(h, steps):
    from oracle.binding import OracleDomain

    o = OracleDomain(h)
    o.run(1, steps)
    F = o.get_fields()[0]
    assert np.all(np.isfinite(F))
    return o, F


def test_gp229_slip_weakening_rupture():
    h = init_domain(_text("gp229/gp229sw3ex1.in"))
    assert (h.mode, h.nx, h.ny, h.nblocks, h.nifaces) == (3, 801, 802, 2, 1)
    # forced nucleation: the tips at x = +-0.76 km close at 1 km/s, so the
    # fault is forced to slip after t = 0.76 s (step 53 at dt = 0.0144 s)
    o, F = _oracle_steps(h, 70)
    V = o.get_fault(0, "V")
    assert V.max() > 0.1 and np.count_nonzero(V) < 40


def test_kali_rate_and_state_with_side_files(tmp_path):
    # kali_input.m: friction parameters, state and prestress along the fault
    y = np.linspace(-30.0, 0.0, 301)
    (tmp_path / "problems").mkdir()
    a = 0.01 + 0.005 * np.sin(2 * np.pi * y / 10)
    b = 0.016 + 0.004 * np.exp(-0.5 * ((y + 15) / 3) ** 2)
    fr = [a, b, 1e-6 + 0 * y, 0.6 + 0 * y, 0.05 + 0 * y, 0 * y, 1e10 + 0 * y]
    np.concatenate(fr).tofile(tmp_path / "problems" / "kali.friction")
    (0.6 + 0.1 * np.exp(y / 5)).tofile(tmp_path / "problems" / "kali.state")
    np.concatenate([np.cos(2 * np.pi * y / 10), np.sin(2 * np.pi * y / 4)]).tofile(tmp_path / "problems" / "kali.prestress")
    h = init_domain(_text("problems/kali-heterogeneous-input.in"), tmp_path)
    assert (h.mode, h.nx, h.ny, h.nifaces) == (3, 602, 301, 1)
    from oracle.binding import OracleDomain

    assert np.array_equal(OracleDomain(h).get_fault(0, "Psi"), 0.6 + 0.1 * np.exp(y / 5))  # state file
    o, F = _oracle_steps(h, 5)
    V = o.get_fault(0, "V")  # locked below y = -25 km (xlockm), creeping above
    assert np.all(np.isfinite(V)) and np.all(V >= 0) and np.count_nonzero(V) > 200


def test_pointsource_layered_medium(tmp_path):
    text = _text("problems/pointsource.in")
    # pointsource_heterogeneous.m: layered rho, cs, cp by depth on the run's own grid
    grid = init_domain(re.sub(r"heterogeneous\s*=\s*true", "heterogeneous = false", text, flags=re.I), tmp_path)
    yy = grid.array("y")[0]
    rho = np.where(yy < -7, 2.8, np.where(yy < -3, 2.3, np.where(yy < -1.5, 1.5, 1.0)))
    cs = np.where(yy < -7, 3.464, np.where(yy < -3, 2.7, np.where(yy < -1.5, 1.0, 0.8)))
    cp = np.where(yy < -7, 6.0, np.where(yy < -3, 5.0, np.where(yy < -1.5, 4.0, 3.6)))
    (tmp_path / "problems").mkdir()
    np.concatenate([rho.ravel(), cs.ravel(), cp.ravel()]).tofile(tmp_path / "problems" / "point_heterogeneous")
    h = init_domain(text, tmp_path)
    assert (h.mode, h.nx, h.ny, h.nblocks, h.heterogeneous) == (2, 201, 52, 2, True)
    o, F = _oracle_steps(h, 40)
    assert np.abs(F[2]).max() > 0  # the Ricker moment tensor source radiates


def test_llw_gaussian_forcing_two_ways(tmp_path):
    """LLWgaussian1 (problem='Forcing') and LLWgaussian2 (the same Gaussian
    from a file, LLWgaussianForcing.m) give the same waves up to the linear
    interpolation of the file's frames in time."""
    h1 = init_domain(_text("problems/LLWgaussian1.in"), tmp_path)
    (tmp_path / "problems").mkdir()
    X = np.arange(-50.0, 51.0)
    x, y = np.meshgrid(X, X)  # (ny, nx), x fastest
    problems.write_forcing_file(tmp_path / "problems" / "LLWgaussian.forcing", x, y, np.arange(101) * 1.25, 3, 0,
                                lambda x, y, t: np.exp(-0.5 * (x / 1.25) ** 2 - 0.5 * (y / 1.25) ** 2)
                                * np.exp(-0.5 * ((t - 8.0) / 2.0) ** 2) / (2.0 * np.sqrt(2 * np.pi)))
    h2 = init_domain(_text("problems/LLWgaussian2.in"), tmp_path)
    assert h1.dt == h2.dt and abs(h1.dt - 1.25) < 1e-12
    _, F1 = _oracle_steps(h1, 30)
    _, F2 = _oracle_steps(h2, 30)
    assert np.abs(F1[0]).max() > 0
    assert np.abs(F1 - F2).max() < 0.05 * np.abs(F1).max()
