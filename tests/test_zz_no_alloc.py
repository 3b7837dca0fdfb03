"""fdmap_gpu_fault_max_noalloc (static device scratch, no allocation) against
the existing read-back path fdmap_gpu_get_fault, on two calls in a row.

Cases: a fault shorter than one CTA's share (one partial), faults of 2561
nodes (three CTAs, so the last CTA folds the other CTAs' partials) with the
maximum planted in each CTA in turn, a NaN planted in the field (the result is
NaN, as np.max of the read-back field is), and a fault of 1,048,577 nodes,
one more than the static scratch covers, which is refused before any launch."""
from __future__ import annotations

import math

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems

pytestmark = pytest.mark.gpu


def test_fault_max_noalloc_matches_get_fault(require_gpu):
    h = init_domain(problems.rupture_sw(nx=81, ny=41, h=0.5, nt=200))
    g = GpuDomain(h)
    for call in range(2):
        g.run(1 + 40 * call, 40 * (call + 1))
        for field in ("V", "S", "N", "D", "DDs", "trup"):
            expect = float(np.max(np.abs(g.get_fault(0, field))))
            got = g.fault_max_noalloc(0, field)
            assert got == pytest.approx(expect, rel=1e-15, abs=0.0), f"call {call}, {field}"
    # a second handle on the same device shares the scratch; calls in sequence are fine
    g2 = GpuDomain(h)
    assert g2.fault_max_noalloc(0, "S") == pytest.approx(float(np.max(np.abs(g2.get_fault(0, "S")))), rel=1e-15)


def test_fault_max_noalloc_several_ctas(require_gpu):
    """2561 fault nodes: three CTAs of 1024 nodes; the maximum sits in the
    first, the middle and the last CTA in turn, each checked on two calls in a
    row (the completion counter starts from zero on every call)."""
    h = init_domain(problems.rupture_sw(nx=2561, ny=9, h=0.05, nt=50))
    g = GpuDomain(h)
    n = h.iface_n(0)
    assert n == 2561
    g.run(1, 10)
    V = g.get_fault(0, "V")
    base = np.abs(V).max()
    for k in (3, 1500, n - 1):
        W = V.copy()
        W[k] = -(10.0 * base + 7.0)  # |.| is the maximum
        g.set_fault(0, "V", W)
        for call in range(2):
            assert g.fault_max_noalloc(0, "V") == float(np.max(np.abs(g.get_fault(0, "V")))) == 10.0 * base + 7.0, \
                f"node {k}, call {call}"
    g.set_fault(0, "V", V)
    for call in range(2):
        assert g.fault_max_noalloc(0, "V") == float(np.max(np.abs(V)))
    # a NaN anywhere makes the maximum NaN, as it does for the read-back field
    for k in (0, n - 1):
        W = V.copy()
        W[k] = np.nan
        g.set_fault(0, "V", W)
        assert math.isnan(float(np.max(np.abs(g.get_fault(0, "V")))))
        assert math.isnan(g.fault_max_noalloc(0, "V")), f"NaN at node {k} was dropped"
    g.set_fault(0, "V", V)
    assert g.fault_max_noalloc(0, "V") == float(np.max(np.abs(V)))


def test_fault_max_noalloc_rejects_bad_arguments(require_gpu):
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=3))
    g = GpuDomain(h)
    with pytest.raises(FdmapError):
        g.fault_max_noalloc(3, "V")


def _long_fault_text(n: int) -> str:
    """Mode III, two blocks of n x 3 nodes (SBP2) joined at a slip-weakening fault y = 0 of n nodes."""
    h = 0.01
    L = (n - 1) * h
    blk = "&material_list rho=2.67d0, cs=3.464d0 /\n&fields_list syy0=-100d0, syz0=50d0 /\n"
    return f"""&problem_list name='long_fault', nt=3, CFL=0.5d0, RKorder=4 /
&domain_list mode=3, FDmethod='SBP2', nblocks_x=1, nblocks_y=2 /
!---BLOCK1---
&grid_list nx={n}, ny=3, LB=0d0,-0.02d0, LT=0d0,0d0, RB={L!r}d0,-0.02d0, RT={L!r}d0,0d0 /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='absorbing', bcT='none' /
{blk}!---BLOCK2---
&grid_list nx={n}, ny=3, LB=0d0,0d0, LT=0d0,0.02d0, RB={L!r}d0,0d0, RT={L!r}d0,0.02d0 /
&boundaries_list bcL='absorbing', bcR='absorbing', bcB='none', bcT='absorbing' /
{blk}!---IFACE1---
&interface_list coupling='friction' /
&friction_list friction_law='SW', sw%fs=0.68d0, sw%fd=0.52d0, sw%Dc=0.4d0 /
"""


def test_fault_max_noalloc_rejects_fault_beyond_scratch(require_gpu):
    """1,048,577 nodes need 1025 partials, one more than the static array
    holds: FDMAP_ERR_UNSUPPORTED (-6) from the host-side size check, and the
    handle keeps working."""
    n = 1024 * 1024 + 1
    h = init_domain(_long_fault_text(n))
    assert h.iface_n(0) == n
    g = GpuDomain(h)
    with pytest.raises(FdmapError) as e:
        g.fault_max_noalloc(0, "S")
    assert e.value.code == -6
    assert float(np.max(np.abs(g.get_fault(0, "S")))) > 0.0
    g.close()
