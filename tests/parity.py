"""Shared helpers for GPU-vs-oracle parity tests.

Tolerances (FP64 throughout):
  FIELD_RTOL  body fields and rates: max|gpu - oracle| / max|oracle| per field
  FAULT_RTOL  fault slip, slip rate, stress, state: same norm-wise measure.  The
              fault solve stops at the reference's residual tolerance
              atolR = 1e4*eps MPa (friction.f90:931), so the GPU's and the
              oracle's iterates may differ at that level each stage.
  Rupture times are step-quantised threshold crossings; they must agree
  exactly at all but a few nodes and within one time step everywhere.
"""
from __future__ import annotations

import numpy as np

FIELD_RTOL = 1e-10
FAULT_RTOL = 1e-8


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


def assert_fault_close(gpu, orc, iface=0, rtol=FAULT_RTOL, dt=None, fields=("V", "S", "N", "D", "Psi")):
    out = fault_errors(gpu, orc, iface, fields)
    for f, e in out.items():
        assert e <= rtol, f"fault {f}: relative error {e} exceeds {rtol}"
    tg, to = gpu.get_fault(iface, "trup"), orc.get_fault(iface, "trup")
    mismatch = np.count_nonzero(tg != to)
    assert mismatch <= max(2, tg.size // 500), f"rupture time differs at {mismatch} of {tg.size} nodes"
    if dt is not None and mismatch:
        both = (tg < 1e9) & (to < 1e9)
        assert np.max(np.abs(tg[both] - to[both]), initial=0.0) <= dt * (1 + 1e-12)
    out["trup_mismatch"] = mismatch
    return out
