"""GPU against the oracle on the benchmarked configurations at their full
grid sizes:

  rupture     two blocks of 1601 x 801 nodes (dx 25 m), slip-weakening fault
              of 1601 nodes, LS-RK4 at CFL 0.5 (the bench workload)
  roughfault  two curvilinear blocks of 2001 x 1001 nodes on a seeded fractal
              fault of 2001 nodes, flash-heating rate-and-state (RFL)

By default 300 steps of the rupture and 50 of the rough fault (about half a
minute and two minutes of the oracle on 16 host cores; 200 rough-fault steps
take ten, set FDMAP_ROUGH_STEPS to run them).  With FDMAP_FULL_LENGTH=1 the
whole runs, 4000 and 6000 steps (nt = 4001 and 6001 loop indices, the last
one the reference's output-only index), are compared instead.  Every case prints one line
`FULLSIZE {json}` with the per-field and fault errors and the tolerances
they were held to (tests/parity.py: 1e-10 for the slip-weakening rupture; for
the rate-and-state run the spread of the oracle's own answer when its Newton
tolerance is halved, measured in the same test)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from tests.parity import FIELD_RTOL, assert_fault_close, assert_fields_close, fault_errors, field_errors, law_tolerances

pytestmark = pytest.mark.gpu

FULL = os.environ.get("FDMAP_FULL_LENGTH") == "1"


def _compare(name, h, n_last, law, fault_fields=("V", "S", "N", "D", "Psi")):
    from oracle.binding import OracleDomain

    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, n_last)
    o.run(1, n_last)
    Fg, Fo = g.get_fields()[0], o.get_fields()[0]
    ferr = field_errors(Fg, Fo)
    flt = fault_errors(g, o, fields=fault_fields)
    tg, to = g.get_fault(0, "trup"), o.get_fault(0, "trup")
    # explicit solves: 1e-10; rate-and-state: the spread within the reference's solver tolerance
    ftol, qtol = law_tolerances(law, h, n_last, fault_fields, base=o)
    rec = {"case": name, "nx": h.nx, "ny": h.ny, "loop_indices": n_last, "field_rel_err": ferr,
           "fault_rel_err": flt, "field_tolerance": ftol, "fault_tolerance": qtol,
           "trup_mismatch_nodes": int(np.count_nonzero(tg != to)),
           "max_slip_rate": float(np.abs(o.get_fault(0, "V")).max()),
           "newton": [g.newton_failures(), o.newton_failures()]}
    print("FULLSIZE " + json.dumps(rec), flush=True)
    assert_fields_close(Fg, Fo, rtol=ftol, what=name)
    assert_fault_close(g, o, rtol=qtol, dt=h.dt, fields=fault_fields)
    g.close()
    o.close()
    return rec


def test_rupture_full_grid(require_gpu):
    h = init_domain(problems.rupture_sw())
    assert (h.nx, h.ny) == (1601, 1602)
    rec = _compare("rupture 2x1601x801", h, h.nt if FULL else 300, "SW", ("V", "S", "N", "D"))
    assert rec["max_slip_rate"] > 0.1  # the patch has nucleated


def test_roughfault_full_grid(require_gpu, tmp_path):
    h = init_domain(problems.rough_fault_rs(tmp_path), tmp_path)
    assert (h.nx, h.ny) == (2001, 2002)
    steps = int(os.environ.get("FDMAP_ROUGH_STEPS", "50"))
    _compare("roughfault 2x2001x1001", h, h.nt if FULL else steps, "RFL")


def test_field_tolerance_is_the_stated_one():
    assert FIELD_RTOL == 1e-10
