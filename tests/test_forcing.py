"""Source forcing terms of set_source (source.f90:147-324) beyond the point
source: the long-wave 'Forcing' problem (Gaussian in space and time, mode III)
and forcing read from a file, one frame per step, interpolated linearly in
time.  Known answers on the oracle, then the GPU against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuAdjoint, GpuDomain, init_domain, problems
from tests.parity import assert_fields_close


def _gauss(amp=1.0, sigma=1.25, sigmat=2.0):
    return lambda x, y, t: (amp * np.exp(-0.5 * (x / sigma) ** 2 - 0.5 * (y / sigma) ** 2)
                            * np.exp(-0.5 * ((t - 4 * sigmat) / sigmat) ** 2) / (sigmat * np.sqrt(2 * np.pi)))


def _forcing_file(tmp_path, h, frames, fn, name="g.forcing"):
    x, y = h.array("x")[0], h.array("y")[0]
    path = tmp_path / name
    problems.write_forcing_file(path, x, y, [h.t0 + k * h.dt for k in range(frames)], h.nF, 0, fn)
    return path


def test_gaussian_forcing_stage_rates():
    """From rest, the first stage rates are the forcing term itself."""
    from oracle.binding import OracleDomain

    h = init_domain(problems.gaussian_forcing(n=41, L=40.0))
    o = OracleDomain(h)
    o.time_step_LS(h.t0, h.dt, True)
    DF = o.get_fields(False, True)[1]
    ref = _gauss()(h.array("x")[0], h.array("y")[0], h.t0)
    np.testing.assert_allclose(DF[0], ref, rtol=1e-14, atol=1e-300)
    assert not np.any(DF[1:])


def test_forcing_file_frames_and_interpolation(tmp_path):
    """Step 1 starts from frame 0 (weights 1, 0); stage rates interpolate the
    frames of the step linearly in time, so frames linear in t reproduce t."""
    from oracle.binding import OracleDomain

    h0 = init_domain(problems.gaussian_forcing(n=21, L=20.0))
    path = _forcing_file(tmp_path, h0, 6, lambda x, y, t: (1.0 + x * x) * t)
    h = init_domain(problems.gaussian_forcing(n=21, L=20.0, forcing_file=str(path)))
    o = OracleDomain(h)
    o.time_step_LS(h.t0, h.dt, True)
    DF = o.get_fields(False, True)[1]
    x = h.array("x")[0]
    assert np.array_equal(DF[0], (1.0 + x * x) * h.t0)
    # a second domain stepped once, then stage 1 of step 2 sees frames 1 and 2
    o2 = OracleDomain(h)
    o2.time_step_LS(h.t0, h.dt)
    o2.set_fields(np.zeros((h.nF, h.ny, h.nx)), None)
    o2.time_step_LS(h.t0 + h.dt, h.dt, True)
    DF2 = o2.get_fields(False, True)[1]
    np.testing.assert_allclose(DF2[0], (1.0 + x * x) * (h.t0 + h.dt), rtol=1e-14)


def test_file_forcing_approximates_the_gaussian_forcing(tmp_path):
    """The same Gaussian sampled once per step (as a forcing file) drives the
    same waves up to the linear-interpolation error in time."""
    from oracle.binding import OracleDomain

    ha = init_domain(problems.gaussian_forcing(n=81, L=40.0, sigma=3.0, sigmat=4.0))
    path = _forcing_file(tmp_path, ha, ha.nt + 1, _gauss(sigma=3.0, sigmat=4.0))
    hb = init_domain(problems.gaussian_forcing(n=81, L=40.0, sigma=3.0, sigmat=4.0, forcing_file=str(path)))
    oa, ob = OracleDomain(ha), OracleDomain(hb)
    oa.run(1, 40)
    ob.run(1, 40)
    Fa, Fb = oa.get_fields()[0], ob.get_fields()[0]
    assert np.abs(Fa[0]).max() > 0
    assert np.abs(Fa - Fb).max() < 0.02 * np.abs(Fa).max()


@pytest.mark.gpu
def test_forcing_file_missing(require_gpu, tmp_path):
    h = init_domain(problems.gaussian_forcing(n=21, L=20.0, forcing_file=str(tmp_path / "absent.forcing")))
    with pytest.raises(FdmapError) as e:
        GpuDomain(h)
    assert e.value.code == -7


def test_adjoint_rejects_forcing(tmp_path):
    text = problems.heterogeneous_ricker(tmp_path, n=31, h=0.1, nt=5)
    text = text.replace("&source_list", "&source_list problem='Forcing', gauss_amp=1d0, gauss_sigma=1d0, gauss_sigmat=1d0,")
    h = init_domain(text, tmp_path)
    with pytest.raises(FdmapError) as e:
        GpuAdjoint(h, [(5, 31)])
    assert e.value.code == -6


# ---------------------------------------------------------------- GPU

@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["gauss", "file"])
@pytest.mark.parametrize("graphs", [True, False])
def test_gpu_forcing_vs_oracle(require_gpu, tmp_path, kind, graphs):
    from oracle.binding import OracleDomain

    h = init_domain(problems.gaussian_forcing(n=81, L=40.0, sigma=3.0, sigmat=4.0))
    if kind == "file":
        path = _forcing_file(tmp_path, h, h.nt + 1, _gauss(sigma=3.0, sigmat=4.0))
        h = init_domain(problems.gaussian_forcing(n=81, L=40.0, sigma=3.0, sigmat=4.0, forcing_file=str(path)))
    g = GpuDomain(h)
    o = OracleDomain(h)
    steps = 30
    if graphs:
        g.run(1, steps)
    else:
        for n in range(1, steps + 1):
            g.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
    o.run(1, steps)
    Fg, Fo = g.get_fields()[0], o.get_fields()[0]
    assert np.abs(Fo).max() > 0
    assert_fields_close(Fg, Fo)
    g.close()


@pytest.mark.gpu
def test_gpu_file_forcing_mode2_with_point_source(require_gpu, tmp_path):
    """Mode II: every field of a frame enters its rate (szz after rates_szz)."""
    from oracle.binding import OracleDomain

    h0 = init_domain(problems.pml_pulse(n=41, L=4.0, width=0.5, sigma=0.0, bc="absorbing"))
    x, y = h0.array("x")[0], h0.array("y")[0]
    path = tmp_path / "m2.forcing"
    with open(path, "wb") as f:
        for k in range(30):
            t = h0.t0 + k * h0.dt
            frame = np.stack([np.sin(x + l + t) * np.cos(y - t) for l in range(h0.nF)])
            frame.tofile(f)
    text = problems.pml_pulse(n=41, L=4.0, width=0.5, sigma=0.0, bc="absorbing").split("&pml_list")[0]
    text += f"&source_list forcing_from_file=T, forcing_filename='{path}' /\n"
    h = init_domain(text)
    g, o = GpuDomain(h), OracleDomain(h)
    g.run(1, 20, nt=1 << 30)
    o.run(1, 20, nt=1 << 30)
    assert_fields_close(g.get_fields()[0], o.get_fields()[0])
    g.close()
