"""Two-stage passes (march_pair.cuh): stages (1,2), (3,4) of every LS-RK4 step
run as one interior pass each, with the boundary work of both stages beside
and after it.  Every node's arithmetic is the stage-by-stage arithmetic (the
same split_rates routine, the same closure and interface code), so a run with
passes must equal the run stage by stage bit for bit: fields, rates and all 18
fault fields.  Cases cover mode II and III, SBP2 and SBP4, faults normal to y
and to x, rate-and-state and slip weakening, a locked interface, every outer
boundary condition, RK orders 2 and 3 (odd and even pair counts), eager steps
and CUDA-graph steps, serialised (profiling) and overlapped launches, blocks
of one strip and of several, CTAs that own one row group and CTAs that own
many, outputs open, and the oracle on the bench workload's shape."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems
from fdmap_github_b200.native import FAULT_FIELDS
from tests.parity import assert_fault_close, assert_fields_close
from tests.test_parity_matrix import fault_text

pytestmark = pytest.mark.gpu


def _state(g, nif):
    F, DF = g.get_fields(True, True)
    flt = []
    for k in range(nif):
        try:
            flt += [g.get_fault(k, f) for f in FAULT_FIELDS]
        except FdmapError:  # a locked interface keeps no fault fields
            pass
    return F, DF, flt


def _same(a, b, what):
    Fa, DFa, fa = a
    Fb, DFb, fb = b
    assert np.array_equal(Fa, Fb), f"{what}: fields differ (max {np.max(np.abs(Fa - Fb)):.3e})"
    assert np.array_equal(DFa, DFb), f"{what}: rates differ (max {np.max(np.abs(DFa - DFb)):.3e})"
    for k, (x, y) in enumerate(zip(fa, fb)):
        assert np.array_equal(x, y, equal_nan=True), f"{what}: fault field {FAULT_FIELDS[k % 18]} differs"


CASES = {
    "II-SW-161x81": lambda: problems.rupture_sw(nx=161, ny=81, h=0.25, nt=61),
    "II-SW-SBP2": lambda: problems.rupture_sw(nx=161, ny=81, h=0.25, nt=61, fd="SBP2"),
    "II-SW-600x300": lambda: problems.rupture_sw(nx=600, ny=300, h=0.1, nt=41),
    "II-RSL-x": lambda: fault_text(mode=2, law="RSL", direction="x", n=81, nt=41),
    "III-RAL": lambda: fault_text(mode=3, law="RAL", n=81, nt=41),
    "III-RFL-x-SBP2": lambda: fault_text(mode=3, law="RFL", direction="x", fd="SBP2", n=81, nt=41),
    "II-locked-x": lambda: fault_text(mode=2, direction="x", coupling="locked", n=81, nt=41),
    "II-SW-free": lambda: fault_text(mode=2, law="SW", bc="free", n=81, nt=41),
    "II-SW-rigid": lambda: fault_text(mode=2, law="SW", bc="rigid", n=81, nt=41),
    "III-pulse": lambda: problems.antiplane_pulse(n=161, L=8.0, nt=41),
    "II-SW-RK3": lambda: problems.rupture_sw(nx=161, ny=81, h=0.25, nt=41, rk=3),
    "II-SW-RK2": lambda: problems.rupture_sw(nx=161, ny=81, h=0.25, nt=41, rk=2),
    # a point force in the interior and in the band: the passes' body-force variant
    "III-locked-source": lambda: fault_text(mode=3, coupling="locked", n=81, nt=41)
    + "&source_list x0=0.37d0, y0=-1.61d0, Fz=1d0, source_time_function='Ricker', t_center=0.3d0, t_duration=0.25d0 /\n",
}


@pytest.mark.parametrize("case", list(CASES))
def test_pairs_equal_stage_by_stage(require_gpu, case):
    h = init_domain(CASES[case]())
    g1, g0 = GpuDomain(h), GpuDomain(h)
    assert g1.two_stage, "the domain should take two-stage passes"
    g0.two_stage = False
    assert not g0.two_stage
    n = h.nt - 1
    g1.run(1, n)
    g0.run(1, n)
    _same(_state(g1, h.nifaces), _state(g0, h.nifaces), case)
    # the final step (stage 1 only, issued eagerly) on top of both
    g1.run(h.nt, h.nt)
    g0.run(h.nt, h.nt)
    _same(_state(g1, h.nifaces), _state(g0, h.nifaces), case + " final step")


def test_pairs_eager_and_profiled_steps(require_gpu):
    """Eager steps (no graph) and serialised launches (profiling on) give the
    bits of graph-replayed, overlapped steps."""
    from fdmap_github_b200.native import lib

    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=61))
    ref, eager, prof = GpuDomain(h), GpuDomain(h), GpuDomain(h)
    ref.run(1, 30)
    for n in range(1, 31):
        eager.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
    lib().fdmap_gpu_profile(prof._g, 1)
    prof.run(1, 30)
    lib().fdmap_gpu_profile(prof._g, 0)
    r = _state(ref, 1)
    _same(_state(eager, 1), r, "eager")
    _same(_state(prof, 1), r, "profiled")


def test_pairs_switch_mid_run(require_gpu):
    """Passes switched off and on between steps keep the run bit-identical."""
    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=61))
    a, b = GpuDomain(h), GpuDomain(h)
    b.two_stage = False
    a.run(1, 10)
    a.two_stage = False
    a.run(11, 17)
    a.two_stage = True
    a.run(18, 30)
    b.run(1, 30)
    _same(_state(a, 1), _state(b, 1), "switched")


def test_pairs_with_outputs_open(require_gpu, tmp_path):
    """The stage-1 output point (fault snapshot, body fields) is unchanged by
    the passes: the same files either way."""
    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=41))
    outs = []
    for on in (True, False):
        g = GpuDomain(h)
        g.two_stage = on
        g.output_add("V", 0, 0, FAULT_FIELDS.index("V"), 1, 161, 1, nmin=0, nmax=1 << 30, stride=1)
        g.output_add("S", 0, 0, FAULT_FIELDS.index("S"), 1, 161, 4, nmin=0, nmax=1 << 30, stride=2)
        g.output_add("vx", 1, 0, 0, 1, 161, 8, 1, 162, 8, nmin=0, nmax=1 << 30, stride=3)
        g.output_add("hat", 2, 4 * 0 + 3, 1, 1, 161, 2, nmin=0, nmax=1 << 30, stride=1)
        prefix = tmp_path / ("on" if on else "off")
        g.output_open(str(prefix), ring_steps=8)
        g.run(1, 40)
        g.output_close()
        outs.append([(prefix.parent / f"{prefix.name}_{n}.dat").read_bytes() for n in ("V", "S", "vx", "hat")])
        g.close()
    assert outs[0] == outs[1]


def test_pairs_against_the_oracle(require_gpu):
    """The bench workload's shape (slip-weakening rupture, SBP4) at 401 x 201
    per block, 100 steps with passes, against the oracle at the stated
    tolerances (1e-10 fields and fault)."""
    from oracle.binding import OracleDomain

    h = init_domain(problems.rupture_sw(nx=401, ny=201, h=0.1, nt=101))
    g, o = GpuDomain(h), OracleDomain(h)
    assert g.two_stage
    g.run(1, 100)
    o.run(1, 100)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0], what="pairs vs oracle")
    assert_fault_close(g, o, rtol=1e-10, dt=h.dt, fields=("V", "S", "N", "D"))


def test_pairs_refused_where_they_do_not_apply(require_gpu, tmp_path):
    """Heterogeneous media, dissipation and SBP6 run stage by stage."""
    for text in (problems.rupture_sw(nx=81, ny=41, h=0.5, nt=5, cdiss=0.3),
                 problems.antiplane_pulse(n=61, L=6.0, nt=5, fd="SBP6"),
                 problems.heterogeneous_ricker(tmp_path, n=61, h=0.1, nt=5)):
        h = init_domain(text, tmp_path)
        g = GpuDomain(h)
        assert not g.two_stage
        with pytest.raises(FdmapError) as e:
            g.two_stage = True
        assert e.value.code == -6
        g.run(1, 3)
        g.close()


def test_tuner_chooses_passes_and_keeps_the_bits(require_gpu):
    """The autotuner times every tile with the passes on and off and keeps the
    fastest; whatever it picks, the run is the untuned run bit for bit."""
    for text in (problems.antiplane_pulse(n=201, L=10.0, nt=41), problems.rupture_sw(nx=321, ny=161, h=0.125, nt=41)):
        h = init_domain(text)
        g, ref = GpuDomain(h), GpuDomain(h)
        tile, ms = g.tune(steps=3)
        assert tile in (0, 1, 2, 3) and ms > 0.0
        assert isinstance(g.two_stage, bool)
        g.run(1, 30)
        ref.run(1, 30)
        _same(_state(g, h.nifaces), _state(ref, h.nifaces), f"tuned ({'passes' if g.two_stage else 'stage by stage'})")
