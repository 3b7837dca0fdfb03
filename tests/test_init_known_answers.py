"""Known answers for the initialisation restatement (init_grid, interp_block,
init_grid_partials, init_edges), independent of the oracle.

A block is given by its four sides as FDMAP reads them: the left and right
sides are skewed straight lines between the block corners (line_map,
geometry.f90:70-106), the bottom and top sides are curve files with a
non-uniform point spacing (read_bnd, grid.f90:646-702).  They are the edges
of the polynomial map, in the unit block coordinates s = (i - 1)/(nx - 1),
t = (j - 1)/(ny - 1),

    x(s, t) = a (s + ex s^2) + c t,      y(s, t) = b (t + ey s t) + d s,

which transfinite interpolation (geometry.f90:153-200) reproduces exactly, and
on which the SBP first derivative with unit spacing (diff, fd.f90:42-80) is
exact to rounding: the SBP4 and SBP6 closures are exact for quadratics, and
SBP2's for linear functions (so ex = 0 there).  At every node the restated
grid, its metric terms xq, xr, yq, yr, the Jacobian J = xq yr - xr yq and Ji
(grid.f90:465-618), and on every side the impedances and SAT penalties
M = [rho cs, rho cp, 1 - 2 (cs/cp)^2, H00i cs |grad| / J, H00i cp |grad| / J]
(init_edges, domain.f90:1349-1459) and the outward unit normals are
compared with these closed forms.  The same map, built on the device
(fdmap_desc.body), is compared on the GPU."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import init_domain

H00I = {"SBP2": 2.0, "SBP4": 2.823529411764706, "SBP6": 3.165067037878233}
RHO, CS, CP = 2.67, 3.464, 6.0
A, B, C, D = 12.0, 7.0, 1.5, 0.8  # block extents and skew (km)


def _write_curve(path, x, y, n1, n2):
    np.concatenate([np.asarray(v, dtype=np.float64).ravel() for v in (x, y, n1, n2)]).tofile(path)


def _map(s, t, ex, ey):
    return A * (s + ex * s * s) + C * t, B * (t + ey * s * t) + D * s


def _block_text(tmp_path, nx, ny, fd, ex, ey, body=False) -> str:
    s = np.linspace(0.0, 1.0, nx)
    # bottom side t = 0: tangent (A(1 + 2 ex s), D); outward normal points to -t
    xb, yb = _map(s, 0.0, ex, ey)
    tb = np.stack([A * (1 + 2 * ex * s), np.full(nx, D + 0.0 * s)])
    nb = np.stack([tb[1], -tb[0]]) / np.hypot(tb[0], tb[1])
    _write_curve(tmp_path / "bottom.curve", xb, yb, nb[0], nb[1])
    # top side t = 1, stored with the downward normal (the reader flips T
    # normals to point out of the block, grid.f90:453)
    xt, yt = _map(s, 1.0, ex, ey)
    tt = np.stack([A * (1 + 2 * ex * s), B * ey + D + 0.0 * s])
    nt = np.stack([tt[1], -tt[0]]) / np.hypot(tt[0], tt[1])
    _write_curve(tmp_path / "top.curve", xt, yt, nt[0], nt[1])
    lb, lt = _map(0.0, 0.0, ex, ey), _map(0.0, 1.0, ex, ey)
    rb, rt = _map(1.0, 0.0, ex, ey), _map(1.0, 1.0, ex, ey)
    f = lambda p: f"{p[0]!r}d0,{p[1]!r}d0"  # noqa: E731
    return f"""&problem_list name='analytic_map', nt=3, CFL=0.5d0, RKorder=4 /
&domain_list mode=2, FDmethod='{fd}', nblocks_x=1, nblocks_y=1 /
!---BLOCK1---
&grid_list nx={nx}, ny={ny}, LB={f(lb)}, LT={f(lt)}, RB={f(rb)}, RT={f(rt)},
  bndBfile='bottom.curve', bndTfile='top.curve' /
&boundaries_list bcL='absorbing', bcR='free', bcB='rigid', bcT='absorbing' /
&material_list rho={RHO!r}d0, cs={CS!r}d0, cp={CP!r}d0 /
"""


def expected(nx, ny, ex, ey):
    """Closed forms on the (ny, nx) grid: x, y, xq, xr, yq, yr, J."""
    s = np.linspace(0.0, 1.0, nx)[None, :]
    t = np.linspace(0.0, 1.0, ny)[:, None]
    hs, ht = 1.0 / (nx - 1), 1.0 / (ny - 1)
    x, y = _map(s, t, ex, ey)
    xq = A * (1 + 2 * ex * s) * hs + 0 * t
    xr = C * ht + 0 * s * t
    yq = (B * ey * t + D) * hs + 0 * s
    yr = B * (1 + ey * s) * ht + 0 * t
    return {"x": x, "y": y, "xq": xq, "xr": xr, "yq": yq, "yr": yr, "J": xq * yr - xr * yq}


CASES = [("SBP4", 0.08, 0.12), ("SBP6", 0.08, 0.12), ("SBP2", 0.0, 0.12)]


def _check_host(h, nx, ny, fd, ex, ey, tol=1e-11):
    e = expected(nx, ny, ex, ey)
    for k in ("x", "y"):
        got = h.array(k)[0]
        err = np.max(np.abs(got - e[k])) / np.max(np.abs(e[k]))
        assert err <= 1e-14, f"{fd}: grid {k} off the map by {err}"
    for k in ("xq", "xr", "yq", "yr", "J"):
        got = h.array(k)[0]
        err = np.max(np.abs(got - e[k])) / np.max(np.abs(e[k]))
        assert err <= tol, f"{fd}: metric {k} relative error {err}"
    err = np.max(np.abs(h.array("Ji")[0] * e["J"] - 1.0))
    assert err <= tol, f"{fd}: Ji * J - 1 = {err}"
    return e


def _expected_side_M(e, side, H00i):
    if side in (0, 1):  # L, R: |grad| = |(xr, yr)| at i = 1 or nx
        col = 0 if side == 0 else -1
        g = np.hypot(e["xr"][:, col], e["yr"][:, col]) / e["J"][:, col]
    else:  # B, T: |(xq, yq)| at j = 1 or ny
        row = 0 if side == 2 else -1
        g = np.hypot(e["xq"][row, :], e["yq"][row, :]) / e["J"][row, :]
    n = g.size
    return np.stack([np.full(n, RHO * CS), np.full(n, RHO * CP), np.full(n, 1 - 2 * (CS / CP) ** 2),
                     H00i * CS * g, H00i * CP * g])


def _expected_normals(e, side):
    if side in (0, 1):
        col = 0 if side == 0 else -1
        tx, ty = e["xr"][:, col], e["yr"][:, col]  # tangent along t
        sgn = -1.0 if side == 0 else 1.0
        nrm = np.stack([ty, -tx]) * sgn
    else:
        row = 0 if side == 2 else -1
        tx, ty = e["xq"][row, :], e["yq"][row, :]  # tangent along s
        sgn = 1.0 if side == 2 else -1.0
        nrm = np.stack([ty, -tx]) * sgn
    return nrm / np.hypot(nrm[0], nrm[1])


@pytest.mark.parametrize("fd,ex,ey", CASES)
def test_metrics_and_edges_on_polynomial_map(tmp_path, fd, ex, ey):
    nx, ny = 61, 37
    h = init_domain(_block_text(tmp_path, nx, ny, fd, ex, ey), tmp_path)
    e = _check_host(h, nx, ny, fd, ex, ey)
    for side in range(4):
        M = h.side_array(0, side, "M")
        Me = _expected_side_M(e, side, H00I[fd])
        err = np.max(np.abs(M - Me) / np.abs(Me).max(axis=1, keepdims=True))
        assert err <= 1e-11, f"{fd}: side {side} impedances/penalties relative error {err}"
        nrm = h.side_array(0, side, "normal")
        nerr = np.max(np.abs(nrm - _expected_normals(e, side)))
        assert nerr <= 1e-12, f"{fd}: side {side} outward normal off by {nerr}"


def test_map_is_not_trivial():
    """The map really is curved and skewed: metrics vary over the block and
    the left and right sides are not vertical."""
    e = expected(61, 37, 0.08, 0.12)
    assert np.ptp(e["xq"]) > 0.1 * np.abs(e["xq"]).max()
    assert np.ptp(e["yr"]) > 0.05 * np.abs(e["yr"]).max()
    assert np.abs(e["xr"]).min() > 0 and np.abs(e["yq"]).min() > 0


@pytest.mark.gpu
@pytest.mark.parametrize("fd,ex,ey", CASES[:2])
def test_device_built_metrics_on_polynomial_map(require_gpu, tmp_path, fd, ex, ey):
    """The engine builds the same block on the device (grid, metrics,
    impedances); against the closed forms."""
    from fdmap_github_b200 import GpuDomain

    nx, ny = 61, 37
    h = init_domain(_block_text(tmp_path, nx, ny, fd, ex, ey), tmp_path, body_on_device=True)
    g = GpuDomain(h)
    e = expected(nx, ny, ex, ey)
    for k in ("xq", "xr", "yq", "yr"):
        got = g.get_metric(k)[0] if g.get_metric(k).ndim == 3 else g.get_metric(k)
        err = np.max(np.abs(got - e[k])) / np.max(np.abs(e[k]))
        assert err <= 1e-11, f"{fd}: device metric {k} relative error {err}"
    Ji = g.get_metric("Ji")
    Ji = Ji[0] if Ji.ndim == 3 else Ji
    assert np.max(np.abs(Ji * e["J"] - 1.0)) <= 1e-11
    for side in range(4):
        M = g.get_side_impedance(0, side)
        Me = _expected_side_M(e, side, H00I[fd])
        err = np.max(np.abs(M.reshape(Me.shape) - Me) / np.abs(Me).max(axis=1, keepdims=True))
        assert err <= 1e-11, f"{fd}: device side {side} relative error {err}"
    g.close()
