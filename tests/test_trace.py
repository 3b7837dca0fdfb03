"""Kernel timeline (fdmap_gpu_trace): one record per CTA of the stage kernels."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems

pytestmark = pytest.mark.gpu


def test_trace_records_every_stage_kernel(require_gpu):
    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=50))
    g = GpuDomain(h)
    g.two_stage = False  # stage by stage: one march launch per stage
    g.run(1, 3)
    g.trace(100000)
    g.run(4, 5)  # two steps, five stages each
    r = g.trace_records()
    kinds = set(r[:, 0].tolist())
    assert kinds == {1, 2, 3}, kinds
    assert np.all(r[:, 4] >= r[:, 3])
    march = r[r[:, 0] == 1]
    assert len(march) % 10 == 0 and len(march) // 10 >= 1  # every CTA of every stage launch
    g.trace(0)
    g.run(6, 7)
    assert len(g.trace_records()) == len(r)  # off: nothing more is recorded
    # the traced run is the same run
    ref = GpuDomain(h)
    ref.run(1, 7)
    assert np.array_equal(ref.get_fields()[0], g.get_fields()[0])


def test_trace_records_two_stage_passes(require_gpu):
    """With two-stage passes a step is two passes (kind 5), their bands (6),
    the single fifth stage (1), and the closure and interface kernels."""
    h = init_domain(problems.rupture_sw(nx=161, ny=81, h=0.25, nt=50))
    g = GpuDomain(h)
    assert g.two_stage
    g.run(1, 3)
    g.trace(100000)
    g.run(4, 5)
    r = g.trace_records()
    assert set(r[:, 0].tolist()) == {1, 2, 3, 5, 6}
    grid = len(set(r[r[:, 0] == 5][:, 2].tolist()))
    assert len(r[r[:, 0] == 5]) == 4 * grid  # two passes a step, every CTA
    assert len(r[r[:, 0] == 1]) % 2 == 0
