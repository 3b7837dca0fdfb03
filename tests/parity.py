"""Shared helpers for GPU-vs-oracle parity tests.

Tolerances (FP64 throughout; errors are max|gpu - oracle| / max|oracle| per
field, the body fields scaled per physical group):

  FIELD_RTOL  1e-10 on the body fields.
  FAULT_RTOL  1e-10 on the fault fields where the interface solve is explicit:
              slip weakening, frictionless, locked, forced rupture.
  Rate-and-state laws: the reference stops its Newton iteration once the
              residual is below atolR = 1e4*eps MPa (friction.f90:931), so its
              own answer is only fixed to within what that tolerance lets
              through, and strongly rate-weakening laws (flash heating)
              amplify that spread along the run.  The bound is measured, not
              guessed: solver_spread() runs the oracle a second time with
              atolR halved; every field and fault field of the GPU must lie
              within SPREAD_FACTOR times that spread (and never needs to be
              closer than 1e-10).  On a 41 x 42 flash-heating rupture after
              200 steps the spread is 5e-6 on the fields; on the aging law
              after 30 steps it is 1e-13.
  Rupture times are step-quantised threshold crossings; they must agree
  exactly at all but a few nodes and within one time step everywhere.
"""
from __future__ import annotations

import numpy as np

FIELD_RTOL = 1e-10
FAULT_RTOL = 1e-10
SPREAD_FACTOR = 2.0
EXPLICIT_LAWS = {"SW", "frictionless", "locked", None}


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    scale = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(a - b)))
    if scale == 0.0:
        return d
    return d / scale


def field_groups(nF: int) -> list[list[int]]:
    """Fields sharing a physical scale: velocities and stresses."""
    return [[0, 1], [2, 3, 4, 5]] if nF == 6 else [[0], [1, 2]]


def field_errors(Fg: np.ndarray, Fo: np.ndarray) -> list[float]:
    """Per-field max error, scaled by the largest magnitude in the field's
    group (a field that is identically zero up to round-off, such as a rate of a
    uniform stress component, is measured against its physical scale)."""
    errs = [0.0] * Fo.shape[0]
    for grp in field_groups(Fo.shape[0]):
        scale = max(float(np.max(np.abs(Fo[l]))) for l in grp)
        for l in grp:
            d = float(np.max(np.abs(Fg[l] - Fo[l])))
            errs[l] = d / scale if scale > 0 else d
    return errs


def assert_fields_close(Fg, Fo, rtol=FIELD_RTOL, what="F"):
    errs = field_errors(Fg, Fo)
    assert np.all(np.isfinite(Fg)), f"{what}: non-finite values on the GPU"
    assert max(errs) <= rtol, f"{what}: per-field relative errors {errs} exceed {rtol}"
    return errs


def fault_errors(gpu, orc, iface=0, fields=("V", "S", "N", "D", "Psi")) -> dict:
    """Norm-wise relative error of each fault field (GPU against oracle)."""
    out = {}
    for f in fields:
        g, o = gpu.get_fault(iface, f), orc.get_fault(iface, f)
        assert np.all(np.isfinite(g)), f"fault {f}: non-finite"
        out[f] = rel_err(g, o)
    return out


def solver_spread(host, n_last, fields=("V", "S", "N", "D", "Psi"), iface=0, base=None, **run_kw):
    """How far the oracle's own result moves when its Newton residual
    tolerance atolR is halved: (largest field error, {fault field: error}).
    `base`: an oracle already run over the same loop indices at the
    reference's tolerance, used in place of a fresh run."""
    from oracle.binding import OracleDomain

    a = base
    if a is None:
        a = OracleDomain(host)
        a.run(1, n_last, **run_kw)
    b = OracleDomain(host)
    b.set_newton_tolerance(0.5)
    b.run(1, n_last, **run_kw)
    fe = max(field_errors(b.get_fields()[0], a.get_fields()[0]))
    ft = fault_errors(b, a, iface, fields) if host.nifaces else {}
    if base is None:
        a.close()
    b.close()
    return fe, ft


def law_tolerances(law, host=None, n_last=None, fields=("V", "S", "N", "D", "Psi"), base=None, **run_kw):
    """(field tolerance, {fault field: tolerance}) for a run with friction law
    `law`: 1e-10 for explicit interface solves; for rate-and-state laws
    SPREAD_FACTOR times the spread within the reference's solver tolerance
    (never below 1e-10)."""
    if law in EXPLICIT_LAWS:
        return FIELD_RTOL, {f: FAULT_RTOL for f in fields}
    fe, ft = solver_spread(host, n_last, fields, base=base, **run_kw)
    return (max(FIELD_RTOL, SPREAD_FACTOR * fe), {f: max(FAULT_RTOL, SPREAD_FACTOR * ft[f]) for f in fields})


def assert_fault_close(gpu, orc, iface=0, rtol=FAULT_RTOL, dt=None, fields=("V", "S", "N", "D", "Psi")):
    """rtol: one tolerance for every field, or {field: tolerance}."""
    out = fault_errors(gpu, orc, iface, fields)
    for f, e in out.items():
        tol = rtol[f] if isinstance(rtol, dict) else rtol
        assert e <= tol, f"fault {f}: relative error {e} exceeds {tol}"
    tg, to = gpu.get_fault(iface, "trup"), orc.get_fault(iface, "trup")
    mismatch = np.count_nonzero(tg != to)
    assert mismatch <= max(2, tg.size // 500), f"rupture time differs at {mismatch} of {tg.size} nodes"
    if dt is not None and mismatch:
        both = (tg < 1e9) & (to < 1e9)
        assert np.max(np.abs(tg[both] - to[both]), initial=0.0) <= dt * (1 + 1e-12)
    out["trup_mismatch"] = mismatch
    return out


def assert_law_parity(gpu, orc, law, host, n_last, dt=None, fields=("V", "S", "N", "D", "Psi"), what="F",
                      **run_kw):
    """Fields and fault of a run of `n_last` loop indices against the oracle,
    with the tolerances of law_tolerances."""
    if dt is not None:
        run_kw.setdefault("dt", dt)  # the oracle runs of the spread take the compared run's step
    ftol, qtol = law_tolerances(law, host, n_last, fields, **run_kw)
    errs = assert_fields_close(gpu.get_fields()[0], orc.get_fields()[0], rtol=ftol, what=what)
    out = assert_fault_close(gpu, orc, rtol=qtol, dt=dt, fields=fields) if host.nifaces else {}
    return errs, out, ftol, qtol
