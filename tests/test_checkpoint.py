"""Checkpoint/resume in FDMAP's FP64 checkpoint layout: a run resumed from a
checkpoint continues bit for bit, and the files have the reference's sizes."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from fdmap_github_b200.checkpoint import checkpoint_read, checkpoint_write
from fdmap_github_b200.native import FAULT_FIELDS


@pytest.mark.gpu
def test_resume_is_bitwise(require_gpu, tmp_path):
    h = init_domain(problems.rupture_sw(nx=61, ny=31, h=0.4, nt=200))
    a = GpuDomain(h)
    a.run(1, 15)
    name = tmp_path / "rup"
    files = checkpoint_write(a, h, name, 15)
    a.run(16, 40)
    Fa, DFa = a.get_fields(True, True)
    b = GpuDomain(h)
    n = checkpoint_read(b, h, name)
    assert n == 15
    b.run(16, 40)
    Fb, DFb = b.get_fields(True, True)
    assert np.array_equal(Fa, Fb) and np.array_equal(DFa, DFb)
    for f in FAULT_FIELDS:
        assert np.array_equal(a.get_fault(0, f), b.get_fault(0, f)), f
    # file sizes as checkpoint_fields / checkpoint_block_fields / checkpoint_friction lay them out
    sizes = {p.name: p.stat().st_size // 8 for p in files}
    assert sizes["rupF.ckpt15"] == 2 * h.nF * h.nx * h.ny
    assert sizes["rupblock1L.ckpt15"] == (3 * h.nF + 2) * 31
    assert sizes["rupblock2T.ckpt15"] == (3 * h.nF + 2) * 61
    assert sizes["rupiface1side1.ckpt15"] == 18 * h.iface_n(0)
