"""Body displacement (domain_list displacement = T; set_rates_displacement,
fields.f90:1245-1258) and peak ground motion (peak = T; update_fields_peak,
fields.f90:1136-1164): known answers of the oracle, the GPU against the
oracle, checkpoint/resume and the ux / pgv outputs."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from fdmap_github_b200.checkpoint import checkpoint_read, checkpoint_write
from fdmap_github_b200.output import configure_outputs


def _flags(text: str, mode: int) -> str:
    return text.replace(f"&domain_list mode={mode}", f"&domain_list mode={mode}, displacement=T, peak=T")


def _rigid_motion():
    """Uniform velocity vz = 1.5 with traction-free sides: the body translates."""
    text = problems.antiplane_pulse(n=31, L=3.0, nt=50, amp=0.0).replace("absorbing", "free")
    text = text.replace("&fields_list", "&fields_list vz0=1.5d0,")
    return _flags(text, 3)


def test_rigid_translation_displacement():
    from oracle.binding import OracleDomain

    h = init_domain(_rigid_motion())
    o = OracleDomain(h)
    o.run(1, 20, nt=1 << 30)
    U, DU = o.get_displacement()
    # exact up to the rounding of the traction-free hat variables
    assert np.allclose(U, 1.5 * 20 * h.dt, rtol=1e-12, atol=0)
    pgv, pga = o.get_peak()
    assert np.allclose(pgv, 1.5, rtol=1e-12, atol=0) and np.abs(pga).max() < 1e-9


def test_peak_velocity_is_the_running_maximum():
    from oracle.binding import OracleDomain

    h = init_domain(_flags(problems.antiplane_pulse(n=41, L=4.0, nt=60), 3))
    o = OracleDomain(h)
    vmax = np.zeros((h.ny, h.nx))
    for n in range(1, 31):
        F = o.get_fields()[0]
        vmax = np.maximum(vmax, np.abs(F[0]))  # stage 1 sees the step-start velocity
        o.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
    assert np.array_equal(o.get_peak()[0], vmax)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["rupture", "pulse"])
def test_gpu_displacement_and_peak_vs_oracle(require_gpu, case):
    from oracle.binding import OracleDomain

    if case == "rupture":
        h = init_domain(_flags(problems.rupture_sw(nx=61, ny=31, h=0.4, nt=100), 2))
    else:
        h = init_domain(_flags(problems.antiplane_pulse(n=61, L=6.0, nt=100), 3))
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 40)
    o.run(1, 40)
    for a, b, what in zip(g.get_displacement() + g.get_peak(), o.get_displacement() + o.get_peak(),
                          ("U", "DU", "pgv", "pga")):
        scale = np.abs(b).max()
        assert scale > 0, what
        assert np.abs(a - b).max() <= 1e-10 * scale, what
    g.close()


@pytest.mark.gpu
def test_resume_with_displacement_and_peak(require_gpu, tmp_path):
    h = init_domain(_flags(problems.rupture_sw(nx=61, ny=31, h=0.4, nt=100), 2))
    a = GpuDomain(h)
    a.run(1, 12)
    files = checkpoint_write(a, h, tmp_path / "x", 12)
    a.run(13, 30)
    b = GpuDomain(h)
    assert checkpoint_read(b, h, tmp_path / "x") == 12
    b.run(13, 30)
    assert np.array_equal(a.get_fields()[0], b.get_fields()[0])
    for p, q in zip(a.get_displacement() + a.get_peak(), b.get_displacement() + b.get_peak()):
        assert np.array_equal(p, q)
    sizes = {p.name: p.stat().st_size // 8 for p in files}
    assert sizes["xF.ckpt12"] == (2 * h.nF + 2 * 2 + 2) * h.nx * h.ny


@pytest.mark.gpu
def test_displacement_and_peak_outputs(require_gpu, tmp_path):
    text = _flags(problems.antiplane_pulse(n=41, L=4.0, nt=40), 3) + """
!---begin:output_list---
B
body
uz pgv pga
0d0 1d10 2
!---end:output_list---
"""
    h = init_domain(text)
    g = GpuDomain(h)
    configure_outputs(g, h, text, tmp_path / "o", ring_steps=3)
    nsteps = 16
    g.run(1, nsteps, nt=h.nt)
    g.output_close()
    uz = np.fromfile(tmp_path / "o_B_uz.dat", dtype=np.float32).reshape(-1, h.ny, h.nx)
    pgv = np.fromfile(tmp_path / "o_B_pgv.dat", dtype=np.float32).reshape(-1, h.ny, h.nx)
    pga = np.fromfile(tmp_path / "o_B_pga.dat", dtype=np.float32).reshape(-1, h.ny, h.nx)
    assert uz.shape[0] == nsteps // 2
    p = GpuDomain(h)
    for n in range(1, nsteps + 1):
        t0 = h.t0 + (n - 1) * h.dt
        U, _ = p.get_displacement()
        p.time_step_LS(t0, h.dt, final_step=True)  # stage 1: peak updated, nothing advanced
        if (n - 1) % 2 == 0:
            pv, pa = p.get_peak()
            np.testing.assert_array_equal(uz[(n - 1) // 2], U[0].astype(np.float32))
            np.testing.assert_array_equal(pgv[(n - 1) // 2], pv.astype(np.float32))
            np.testing.assert_array_equal(pga[(n - 1) // 2], pa.astype(np.float32))
        p.time_step_LS(t0, h.dt)
    assert np.abs(uz[-1]).max() > 0 and pgv[-1].max() > 0
