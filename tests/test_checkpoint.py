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
    # per side: F, Fhat, F0 per field, U and DU per displacement component (nU = 2), E, DE
    assert sizes["rupblock1L.ckpt15"] == (3 * h.nF + 2 * 2 + 2) * 31
    assert sizes["rupblock2T.ckpt15"] == (3 * h.nF + 2 * 2 + 2) * 61
    assert sizes["rupiface1side1.ckpt15"] == 18 * h.iface_n(0)
    # the boundary displacement resumes too
    for blk in range(2):
        for s in range(4):
            Ua, DUa = a.get_side_displacement(blk, s)
            Ub, DUb = b.get_side_displacement(blk, s)
            assert np.array_equal(Ua, Ub) and np.array_equal(DUa, DUb), (blk, s)
    assert np.abs(a.get_side_displacement(0, 3)[0]).max() > 0  # the fault side has slipped


def test_pml_list_reaches_the_descriptor():
    h = init_domain(problems.pml_pulse(n=41, L=4.0, width=1.0, pmly=False, kappa=0.25, npow=3.0))
    p = h.block_pml(0)
    assert p["pmlx"] and not p["pmly"] and p["n"] == 3.0 and p["kappa"] == 0.25
    assert (p["mx"], p["px"], p["my"], p["py"]) == (1.0, 3.0, 1.0, 3.0)
    assert h.pml_fields() == (True, False)
    q = init_domain(problems.antiplane_pulse(n=21, L=2.0, nt=3)).block_pml(0)
    assert not q["pmlx"] and q["mx"] == -np.finfo(float).max and q["py"] == np.finfo(float).max


@pytest.mark.gpu
def test_resume_with_pml_is_bitwise(require_gpu, tmp_path):
    """The F checkpoint carries Wx and Wy after F and DF (fields.f90:406-407)."""
    h = init_domain(problems.pml_pulse(n=61, L=6.0, width=1.5, nt=200))
    a = GpuDomain(h)
    a.run(1, 25)
    name = tmp_path / "pml"
    files = checkpoint_write(a, h, name, 25)
    a.run(26, 45)
    b = GpuDomain(h)
    assert checkpoint_read(b, h, name) == 25
    b.run(26, 45)
    assert np.array_equal(a.get_fields()[0], b.get_fields()[0])
    assert np.array_equal(a.get_pml("Wx"), b.get_pml("Wx"))
    sizes = {p.name: p.stat().st_size // 8 for p in files}
    assert sizes["pmlF.ckpt25"] == 4 * h.nF * h.nx * h.ny


@pytest.mark.gpu
def test_oracle_resumes_from_gpu_checkpoint(require_gpu, tmp_path):
    """The engine writes the checkpoint files; the oracle reads them (the same
    reader, through the oracle's setters), continues, and lands where its own
    uninterrupted run does."""
    from oracle.binding import OracleDomain

    from tests.parity import assert_fault_close, assert_fields_close

    h = init_domain(problems.rupture_sw(nx=61, ny=31, h=0.4, nt=200))
    g = GpuDomain(h)
    g.run(1, 15)
    name = tmp_path / "rup"
    checkpoint_write(g, h, name, 15)
    b = OracleDomain(h)
    assert checkpoint_read(b, h, name) == 15
    b.run(16, 40)
    a = OracleDomain(h)
    a.run(1, 40)
    assert_fields_close(b.get_fields()[0], a.get_fields()[0], what="resumed F")
    assert_fault_close(b, a, dt=h.dt)
    # boundary displacement of every side, against the largest one (the fault sides)
    sides = [(blk, s) for blk in range(2) for s in range(4)]
    scale = max(float(np.abs(a.get_side_u(blk, s)[0]).max()) for blk, s in sides)
    for blk, s in sides:
        Ub, Ua = b.get_side_u(blk, s)[0], a.get_side_u(blk, s)[0]
        assert np.max(np.abs(Ub - Ua)) <= 1e-10 * scale, (blk, s)
    assert a.get_fault(0, "D").max() > 0.1


def test_oracle_checkpoint_round_trip(tmp_path):
    """The checkpoint writer and reader on the oracle alone (no GPU): resume
    is bit for bit, with the boundary displacement and the fault registers."""
    from oracle.binding import OracleDomain

    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=100))
    a = OracleDomain(h)
    a.run(1, 10)
    checkpoint_write(a, h, tmp_path / "o", 10)
    a.run(11, 20)
    b = OracleDomain(h)
    assert checkpoint_read(b, h, tmp_path / "o") == 10
    b.run(11, 20)
    assert np.array_equal(a.get_fields()[0], b.get_fields()[0])
    for f in FAULT_FIELDS:
        assert np.array_equal(a.get_fault(0, f), b.get_fault(0, f)), f
    assert np.array_equal(a.get_side_u(0, 3)[0], b.get_side_u(0, 3)[0])
