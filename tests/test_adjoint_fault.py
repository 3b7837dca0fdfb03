"""Forward/backward pair across a rate-and-state fault: two heterogeneous mode
III blocks coupled by a frictional (or locked) interface.  The discrete-adjoint
gradient of the receiver misfit with respect to rho(x), G(x) and the shear
prestress S0 of every fault node against central finite differences of the
forward misfit in random directions (h = 1e-6 relative), on the engine's own
forward path (interfaces.f90:676-1012, friction.f90:593-828 for the solve)."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import FdmapError, GpuAdjoint, GpuDomain, init_domain, problems

S0_SCALE = 58.0  # shear stress level of the problem: prestress directions are relative to it


def _setup(tmp_path, law="RAL", coupling="friction", nt=41, K=7, fd="SBP4", seed=1):
    text = problems.heterogeneous_rs_fault(tmp_path, n=41, h=0.25, nt=nt, law=law, fd=fd, seed=seed,
                                           coupling=coupling)
    if coupling == "locked":  # a point force below the interface drives the locked problem
        text += ("&source_list x0=0.37d0, y0=-1.61d0, Fz=1d0, source_time_function='Ricker', "
                 "t_center=0.3d0, t_duration=0.25d0 /\n")
    h = init_domain(text, tmp_path)
    # receivers on rows 2 and 3 nodes off the fault (global rows m and m + 1 are
    # its two edges), where the rupture's waves arrive within the window
    m = h.ny // 2
    cols = np.linspace(3, h.nx - 2, 6).round().astype(int)
    rec = [(int(i), m - 2) for i in cols] + [(int(i), m + 4) for i in cols[::2]]
    return h, rec, GpuAdjoint(h, rec, checkpoint_every=K)


def _material(h):
    return h.array("rho")[0].copy(), h.array("G")[0].copy()


def _data(adj, h):
    """Traces of a perturbed model: a smooth 5 % material bump and a shear
    prestress bump of 2 on the fault."""
    rho, G = _material(h)
    y, x = np.meshgrid(np.linspace(0, 1, h.ny), np.linspace(0, 1, h.nx), indexing="ij")
    bump = np.exp(-((x - 0.4) ** 2 + (y - 0.6) ** 2) / 0.02)
    adj.set_material(rho * (1 + 0.05 * bump), G * (1 - 0.05 * bump))
    nf = adj.fault_size
    s = np.linspace(-1, 1, nf)
    adj.set_prestress(2.0 * np.exp(-((s - 0.2) / 0.3) ** 2))
    d, _ = adj.forward()
    adj.set_material(rho, G)
    adj.set_prestress(np.zeros(nf))
    return d


def test_adjoint_rejects_slip_weakening(tmp_path):
    text = problems.heterogeneous_rs_fault(tmp_path, n=21, h=0.5, nt=5, law="SW")
    text = text.replace("rs%a=0.01d0", "sw%fs=0.68d0, sw%fd=0.52d0, sw%Dc=0.2d0, rs%a=0.01d0")
    h = init_domain(text, tmp_path)
    with pytest.raises(FdmapError) as e:
        GpuAdjoint(h, [(5, h.ny)])
    assert e.value.code == -6


def test_adjoint_rejects_forced_rupture(tmp_path):
    text = problems.heterogeneous_rs_fault(tmp_path, n=21, h=0.5, nt=5)
    text = text.replace("ld%T=0d0 /", "ld%T=0d0, force=T, kn%fd=0.52d0 /")
    h = init_domain(text, tmp_path)
    with pytest.raises(FdmapError) as e:
        GpuAdjoint(h, [(5, h.ny)])
    assert e.value.code == -6


@pytest.mark.gpu
def test_forward_traces_are_the_engine_run(require_gpu, tmp_path):
    h, rec, adj = _setup(tmp_path, nt=31)
    tr, _ = adj.forward()
    g = GpuDomain(h)
    for n in range(1, h.nt + 1):
        F, _ = g.get_fields()
        vz = np.array([F[0, j - 1, i - 1] for i, j in rec])
        assert np.array_equal(vz, tr[n - 1]), f"sample {n}"
        if n < h.nt:
            g.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt)
    assert np.array_equal(adj.fields(), g.get_fields()[0])
    assert np.abs(g.get_fault(0, "V")).max() > 1.0  # the fault ruptures in the window
    g.close()


def _fd_errors(adj, h, data, rng, ndir, what=("rho", "G", "S0"), steps=(1e-6,)):
    """Worst relative error of the adjoint directional derivative against
    central differences, per difference step (relative perturbations)."""
    rho, G = _material(h)
    nf = adj.fault_size
    _, J0 = adj.forward(data=data)
    assert J0 > 0
    g_rho, g_G = adj.backward()
    g_S0 = adj.prestress_gradient()
    assert np.all(np.isfinite(g_rho)) and np.all(np.isfinite(g_G)) and np.all(np.isfinite(g_S0))
    worst = [0.0] * len(steps)
    for _ in range(ndir):
        d_rho = rng.uniform(-1, 1, rho.shape) if "rho" in what else np.zeros_like(rho)
        d_G = rng.uniform(-1, 1, G.shape) if "G" in what else np.zeros_like(G)
        d_S0 = rng.uniform(-1, 1, nf) if "S0" in what else np.zeros(nf)
        pred = float(np.sum(g_rho * rho * d_rho) + np.sum(g_G * G * d_G) + np.sum(g_S0 * S0_SCALE * d_S0))
        for q, eps in enumerate(steps):
            Js = []
            for sgn in (1, -1):
                adj.set_material(rho * (1 + sgn * eps * d_rho), G * (1 + sgn * eps * d_G))
                adj.set_prestress(sgn * eps * S0_SCALE * d_S0)
                Js.append(adj.forward(data=data)[1])
            fd_val = (Js[0] - Js[1]) / (2 * eps)
            worst[q] = max(worst[q], abs(fd_val - pred) / abs(fd_val))
    adj.set_material(rho, G)
    adj.set_prestress(np.zeros(nf))
    return worst, (g_rho, g_G, g_S0)


def _fd_check(adj, h, data, rng, ndir, what=("rho", "G", "S0")):
    worst, grads = _fd_errors(adj, h, data, rng, ndir, what)
    return worst[0], grads


@pytest.mark.gpu
@pytest.mark.parametrize("law", ["RAL", "RSL"])
def test_gradient_vs_central_differences(require_gpu, tmp_path, law):
    rng = np.random.default_rng(17)
    h, rec, adj = _setup(tmp_path, law=law)
    data = _data(adj, h)
    ndir = 16 if law == "RAL" else 6
    worst, (g_rho, g_G, g_S0) = _fd_check(adj, h, data, rng, ndir)
    assert np.any(g_S0 != 0.0)
    assert worst <= 1e-6, f"{law}: adjoint vs central differences, worst relative error {worst:.3e}"


@pytest.mark.gpu
def test_flash_heating_gradient_is_the_difference_limit(require_gpu, tmp_path):
    """With flash heating (RFL) this rupture reaches 20 m/s and the misfit is
    strongly nonlinear in the prestress: central differences at h = 1e-6 still
    carry their O(h^2) truncation error.  They converge onto the adjoint value
    as h shrinks (about 100x per decade of h)."""
    rng = np.random.default_rng(17)
    h, rec, adj = _setup(tmp_path, law="RFL")
    data = _data(adj, h)
    (e6, e7), _ = _fd_errors(adj, h, data, rng, 4, steps=(1e-6, 1e-7))
    assert e7 <= 1e-4, f"RFL: worst relative error {e7:.3e} at h = 1e-7"
    assert e6 <= 1e-6 or e6 / e7 >= 10.0, f"RFL: no convergence, {e6:.3e} (1e-6) -> {e7:.3e} (1e-7)"


@pytest.mark.gpu
def test_prestress_gradient_alone_vs_central_differences(require_gpu, tmp_path):
    """Directions in the prestress only: the part of the gradient that runs
    entirely through the implicit derivative of the friction solve."""
    rng = np.random.default_rng(23)
    h, rec, adj = _setup(tmp_path)
    data = _data(adj, h)
    worst, _ = _fd_check(adj, h, data, rng, 6, what=("S0",))
    assert worst <= 1e-6, f"prestress: worst relative error {worst:.3e}"


@pytest.mark.gpu
def test_locked_interface_gradient(require_gpu, tmp_path):
    rng = np.random.default_rng(29)
    h, rec, adj = _setup(tmp_path, coupling="locked")
    rho, G = _material(h)
    y, x = np.meshgrid(np.linspace(0, 1, h.ny), np.linspace(0, 1, h.nx), indexing="ij")
    adj.set_material(rho * (1 + 0.05 * np.exp(-((x - 0.4) ** 2 + (y - 0.6) ** 2) / 0.02)), G)
    data, _ = adj.forward()
    adj.set_material(rho, G)
    worst, _ = _fd_check(adj, h, data, rng, 4, what=("rho", "G"))
    assert worst <= 1e-6


@pytest.mark.gpu
def test_gradient_independent_of_checkpoint_interval(require_gpu, tmp_path):
    h, rec, a7 = _setup(tmp_path, K=7)
    data = _data(a7, h)
    a7.forward(data=data)
    g7 = a7.backward() + (a7.prestress_gradient(),)
    a80 = GpuAdjoint(h, rec, checkpoint_every=80)
    a80.set_material(*_material(h))  # same edge impedances as a7 (set_material path)
    a80.forward(data=data)
    g80 = a80.backward() + (a80.prestress_gradient(),)
    for x, y in zip(g7, g80):
        assert np.array_equal(x, y)


@pytest.mark.gpu
def test_resident_segments_match_recompute(require_gpu, tmp_path):
    """Fields, state variable and slip rate of resident segments (all, or the
    last two with the rest recomputed after them) give the recomputed
    gradients in rho, G and S0 bit for bit."""
    h, rec, a = _setup(tmp_path, K=7)  # 40 steps: 6 segments
    data = _data(a, h)
    a.forward(data=data)
    ref = a.backward() + (a.prestress_gradient(),)
    seg = a.segment_bytes
    for budget, want in ((-1, 6), (3 * seg, 2)):
        a.set_store_budget(budget)
        a.forward(data=data)
        assert a.resident_segments == want
        for _ in range(2):
            for x, y in zip(ref, a.backward() + (a.prestress_gradient(),)):
                assert np.array_equal(x, y), budget


@pytest.mark.gpu
def test_fault_nodes_carry_material_gradient(require_gpu, tmp_path):
    """The interface impedances depend on rho and G at both edge nodes."""
    h, rec, adj = _setup(tmp_path)
    data = _data(adj, h)
    adj.forward(data=data)
    g_rho, g_G = adj.backward()
    m = h.ny // 2
    for row in (m - 1, m):  # edge rows of the two blocks
        assert np.any(g_G[row] != 0.0) and np.any(g_rho[row] != 0.0)


def test_adjoint_rejects_dissipation(tmp_path):
    """The backward pass has no dissipative terms, so a dissipative block is refused."""
    text = problems.heterogeneous_ricker(tmp_path, n=31, h=0.1, nt=5)
    text = text.replace("&material_list heterogeneous=T", "&operator_list Cdiss=0.2d0 /\n&material_list heterogeneous=T")
    h = init_domain(text, tmp_path)
    assert h.block_cdiss(0) > 0
    with pytest.raises(FdmapError) as e:
        GpuAdjoint(h, [(5, 31)])
    assert e.value.code == -6
