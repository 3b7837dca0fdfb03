"""Forward/backward pair: the discrete-adjoint gradient of the receiver misfit
with respect to rho(x) and G(x) against central finite differences of the
forward misfit in random directions (h = 1e-6 relative), on the engine's own
forward path."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuAdjoint, GpuDomain, init_domain, problems

pytestmark = pytest.mark.gpu


def _setup(tmp_path, n=61, nt=81, fd="SBP4", K=7, seed=3, nrec=8):
    text = problems.heterogeneous_ricker(tmp_path, n=n, h=0.1, nt=nt, fd=fd, seed=seed, f_peak=1.0)
    h = init_domain(text, tmp_path)
    cols = np.linspace(3, n - 2, nrec).round().astype(int)
    rec = [(int(i), n) for i in cols]  # top row (1-based)
    return h, rec, GpuAdjoint(h, rec, checkpoint_every=K)


def _material(h):
    return h.array("rho")[0].copy(), h.array("G")[0].copy()


def _data(adj, h, rng):
    """Traces of a perturbed model (smooth 5 % perturbation)."""
    rho, G = _material(h)
    y, x = np.meshgrid(np.linspace(0, 1, h.ny), np.linspace(0, 1, h.nx), indexing="ij")
    bump = np.exp(-((x - 0.4) ** 2 + (y - 0.7) ** 2) / 0.02)
    adj.set_material(rho * (1 + 0.05 * bump), G * (1 - 0.05 * bump))
    d, _ = adj.forward()
    adj.set_material(rho, G)
    return d


def test_forward_traces_are_the_engine_run(require_gpu, tmp_path):
    h, rec, adj = _setup(tmp_path, nt=41)
    tr, _ = adj.forward()
    g = GpuDomain(h)
    for n in range(1, h.nt + 1):
        F, _ = g.get_fields()
        vz = np.array([F[0, j - 1, i - 1] for i, j in rec])
        assert np.array_equal(vz, tr[n - 1]), f"sample {n}"
        if n < h.nt:
            g.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
    assert np.array_equal(adj.fields(), g.get_fields()[0])


@pytest.mark.parametrize("fd", ["SBP2", "SBP4", "SBP6"])
def test_gradient_vs_central_differences(require_gpu, tmp_path, fd):
    rng = np.random.default_rng(11)
    h, rec, adj = _setup(tmp_path, fd=fd)
    data = _data(adj, h, rng)
    rho, G = _material(h)
    _, J0 = adj.forward(data=data)
    assert J0 > 0
    g_rho, g_G = adj.backward()
    assert np.all(np.isfinite(g_rho)) and np.all(np.isfinite(g_G))
    eps = 1e-6
    worst = 0.0
    ndir = 16 if fd == "SBP4" else 4
    for _ in range(ndir):
        d_rho = rng.uniform(-1, 1, rho.shape)
        d_G = rng.uniform(-1, 1, G.shape)
        pred = float(np.sum(g_rho * rho * d_rho) + np.sum(g_G * G * d_G))
        adj.set_material(rho * (1 + eps * d_rho), G * (1 + eps * d_G))
        _, Jp = adj.forward(data=data)
        adj.set_material(rho * (1 - eps * d_rho), G * (1 - eps * d_G))
        _, Jm = adj.forward(data=data)
        fd_val = (Jp - Jm) / (2 * eps)
        err = abs(fd_val - pred) / abs(fd_val)
        worst = max(worst, err)
    adj.set_material(rho, G)
    assert worst <= 1e-6, f"adjoint vs central differences: worst relative error {worst:.3e}"


def test_gradient_independent_of_checkpoint_interval(require_gpu, tmp_path):
    rng = np.random.default_rng(5)
    h, rec, a7 = _setup(tmp_path, K=7)
    data = _data(a7, h, rng)
    a7.forward(data=data)
    g7 = a7.backward()
    a80 = GpuAdjoint(h, rec, checkpoint_every=80)
    a80.set_material(*_material(h))  # same edge impedances as a7 (set_material path)
    a80.forward(data=data)
    g80 = a80.backward()
    for x, y in zip(g7, g80):
        assert np.array_equal(x, y)


def test_resident_segments_match_recompute(require_gpu, tmp_path):
    """Stage inputs kept resident from the forward pass (every segment, some
    of them, none) give the recomputed gradient bit for bit, also from a
    second backward over the same forward; a material change drops them."""
    rng = np.random.default_rng(5)
    h, rec, a = _setup(tmp_path, K=7)  # 80 steps: 12 segments, the last of 3 steps
    data = _data(a, h, rng)
    tr0, J0 = a.forward(data=data)
    ref = a.backward()
    assert a.resident_segments == 0
    seg = a.segment_bytes
    assert seg >= 7 * 5 * 3 * 8 * h.ny * h.nx  # K steps x 5 stages x 3 padded planes
    for budget, want in ((-1, 12), (4 * seg, 3), (seg, 0), (12 * seg, 12)):
        a.set_store_budget(budget)
        tr, J = a.forward(data=data)
        assert np.array_equal(tr, tr0) and J == J0
        assert a.resident_segments == want, budget
        for _ in range(2):
            for x, y in zip(ref, a.backward()):
                assert np.array_equal(x, y), budget
    a.set_material(*_material(h))
    assert a.resident_segments == 0
    for x, y in zip(ref, a.backward()):
        assert np.array_equal(x, y)


def test_boundary_nodes_carry_gradient(require_gpu, tmp_path):
    """The edge impedances depend on rho and G: boundary-node gradients are
    part of the FD-checked total and must not vanish."""
    rng = np.random.default_rng(2)
    h, rec, adj = _setup(tmp_path)
    data = _data(adj, h, rng)
    adj.forward(data=data)
    g_rho, g_G = adj.backward()
    assert np.any(g_G[-1, :] != 0.0) and np.any(g_rho[-1, :] != 0.0)


def test_device_built_body(require_gpu, tmp_path):
    """With the body built on the device the edge geometry factors come from
    the device metric planes: traces, misfit and gradients equal those of the
    adjoint over the host-built body."""
    text = problems.heterogeneous_ricker(tmp_path, n=61, h=0.1, nt=41, seed=3, f_peak=1.0)
    full = init_domain(text, tmp_path)
    dev = init_domain(text, tmp_path, body_on_device=True)
    rec = [(i, 61) for i in (5, 20, 40, 57)]
    af = GpuAdjoint(full, rec, checkpoint_every=7)
    ad = GpuAdjoint(dev, rec, checkpoint_every=7)
    assert (dev.dt, dev.nt) == (full.dt, full.nt)
    rho, G = _material(full)
    y, x = np.meshgrid(np.linspace(0, 1, full.ny), np.linspace(0, 1, full.nx), indexing="ij")
    af.set_material(rho * (1 + 0.05 * np.exp(-((x - 0.4) ** 2 + (y - 0.7) ** 2) / 0.02)), G)
    data, _ = af.forward()
    for a in (af, ad):
        a.set_material(rho, G)
    tf, Jf = af.forward(data=data)
    td, Jd = ad.forward(data=data)
    assert np.array_equal(tf, td) and Jf == Jd and Jf > 0
    for p, q in zip(af.backward(), ad.backward()):
        assert np.array_equal(p, q)
