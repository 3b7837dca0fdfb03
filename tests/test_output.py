"""Device-side output: the reference's output list, the float32 .dat/.t
files, the stage-1 output point, and drains of the device ring."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, init_domain, problems
from fdmap_github_b200.output import configure_outputs, read_output_list

OUT_LIST = """
!---begin:output_list---
I
iface1
x y
0d0 0d0 1
I
iface1
D V S trup
0d0 1d10 1
B
body
vx sxy
0d0 1d10 4
P
point_body
vy
0d0 1d10 1
20 11
G
grid_iface1
V
0d0 1d10 2
5 10 25
!---end:output_list---
"""


def test_read_output_list():
    items = read_output_list(OUT_LIST)
    assert [it.name for it in items] == ["I", "I", "B", "P", "G"]
    assert items[1].fields == ["D", "V", "S", "trup"] and items[1].stride == 1
    assert items[2].location == "body" and items[2].stride == 4 and items[2].tmax == 1e10
    assert items[3].index == [20, 11]
    assert items[4].location == "grid_iface1" and items[4].index == [5, 10, 25]


def _problem(nt=31):
    return problems.rupture_sw(nx=41, ny=21, h=0.5, nt=nt) + OUT_LIST


@pytest.mark.gpu
def test_outputs_match_stage1_state(require_gpu, tmp_path):
    text = _problem()
    h = init_domain(text)
    g = GpuDomain(h)
    prefix = tmp_path / "rup"
    names = configure_outputs(g, h, text, prefix, ring_steps=7)  # small ring: several drains
    assert "I_V" in names and "G_15_V" in names
    nsteps = 30
    g.run(1, nsteps, nt=h.nt)  # graph replays
    g.output_close()
    # reference trajectory with a stage-1 probe per step (final-step semantics:
    # solve and rates only, nothing updated)
    p = GpuDomain(h)
    nf = h.iface_n(0)
    D = np.fromfile(f"{prefix}_I_D.dat", dtype=np.float32).reshape(-1, nf)
    V = np.fromfile(f"{prefix}_I_V.dat", dtype=np.float32).reshape(-1, nf)
    tr = np.fromfile(f"{prefix}_I_trup.dat", dtype=np.float32).reshape(-1, nf)
    vx = np.fromfile(f"{prefix}_B_vx.dat", dtype=np.float32).reshape(-1, h.ny, h.nx)
    vy = np.fromfile(f"{prefix}_P_vy.dat", dtype=np.float32)
    gv = np.fromfile(f"{prefix}_G_15_V.dat", dtype=np.float32)
    t = np.fromfile(f"{prefix}_I_V.t", dtype=np.float32)
    assert D.shape[0] == V.shape[0] == nsteps and vx.shape[0] == (nsteps - 1) // 4 + 1 and gv.size == nsteps // 2
    np.testing.assert_array_equal(t, (h.t0 + np.arange(nsteps) * h.dt).astype(np.float32))
    for n in range(1, nsteps + 1):
        t0 = h.t0 + (n - 1) * h.dt
        F, _ = p.get_fields()
        Dn = p.get_fault(0, "D")  # before the probe: the step-start slip
        p.time_step_LS(t0, h.dt, final_step=True)
        np.testing.assert_array_equal(D[n - 1], Dn.astype(np.float32))
        np.testing.assert_array_equal(V[n - 1], p.get_fault(0, "V").astype(np.float32))
        np.testing.assert_array_equal(tr[n - 1], p.get_fault(0, "trup").astype(np.float32))
        assert vy[n - 1] == np.float32(F[1, 10, 19])
        if (n - 1) % 4 == 0:
            np.testing.assert_array_equal(vx[(n - 1) // 4], F[0].astype(np.float32))
        if (n - 1) % 2 == 0:
            assert gv[(n - 1) // 2] == np.float32(p.get_fault(0, "V")[14])
        p.time_step_LS(t0, h.dt)
    # static items are written once
    x = np.fromfile(f"{prefix}_I_x.dat", dtype=np.float32)
    assert x.size == nf


@pytest.mark.gpu
def test_outputs_eager_steps_equal_graph_steps(require_gpu, tmp_path):
    text = _problem(nt=13)
    h = init_domain(text)
    a, b = GpuDomain(h), GpuDomain(h)
    configure_outputs(a, h, text, tmp_path / "a", ring_steps=4)
    configure_outputs(b, h, text, tmp_path / "b", ring_steps=100)
    a.run(1, h.nt)  # graphs + final step
    for n in range(1, h.nt + 1):
        b.time_step_LS(h.t0 + (n - 1) * h.dt, h.dt, final_step=(n == h.nt))
    a.output_close()
    b.output_close()
    for nm in ("I_D", "I_V", "I_S", "B_vx", "P_vy"):
        x = np.fromfile(tmp_path / f"a_{nm}.dat", dtype=np.float32)
        y = np.fromfile(tmp_path / f"b_{nm}.dat", dtype=np.float32)
        assert x.size > 0 and np.array_equal(x, y), nm


@pytest.mark.gpu
@pytest.mark.parametrize("ring", [1, 2, 3])
def test_outputs_independent_of_ring_size(require_gpu, tmp_path, ring):
    """Rings copied to the host asynchronously every R/2 output steps (R = 1:
    every step) write the same files as one ring that holds the whole run."""
    text = _problem(nt=21)
    h = init_domain(text)
    a, b = GpuDomain(h), GpuDomain(h)
    configure_outputs(a, h, text, tmp_path / "a", ring_steps=ring)
    configure_outputs(b, h, text, tmp_path / "b", ring_steps=100)
    a.run(1, 9)
    a.output_flush()  # a flush between asynchronous copies
    a.run(10, h.nt)
    b.run(1, h.nt)
    a.output_close()
    b.output_close()
    for nm in ("I_D", "I_V", "I_S", "B_vx", "P_vy"):
        for ext in (".dat", ".t"):
            x = np.fromfile(tmp_path / f"a_{nm}{ext}", dtype=np.float32)
            y = np.fromfile(tmp_path / f"b_{nm}{ext}", dtype=np.float32)
            assert x.size > 0 and np.array_equal(x, y), nm + ext


BND_LIST = """
!---begin:output_list---
S
bndT2
ux uy vx vy sxx syy sxy
0d0 1d10 1
X
bndT2
x y
0d0 0d0 1
L
bndB2
ux vy
0d0 1d10 3
!---end:output_list---
"""


def test_read_boundary_output_list():
    items = read_output_list(BND_LIST)
    assert [it.location for it in items] == ["bndT2", "bndT2", "bndB2"]
    assert items[0].fields == ["ux", "uy", "vx", "vy", "sxx", "syy", "sxy"] and items[2].stride == 3


@pytest.mark.gpu
def test_boundary_outputs_match_stage1_state(require_gpu, tmp_path):
    """bndX locations: boundary displacement at the step start and the stage-1
    hat variables (get_field, domain.f90:763-860), here on the free top of the
    upper block and on the fault side of the same block."""
    text = problems.rupture_sw(nx=41, ny=21, h=0.5, nt=31) + BND_LIST
    h = init_domain(text)
    g = GpuDomain(h)
    prefix = tmp_path / "bnd"
    configure_outputs(g, h, text, prefix, ring_steps=5)
    nsteps = 25
    g.run(1, nsteps, nt=h.nt)
    g.output_close()
    n = 41
    out = {f: np.fromfile(f"{prefix}_S_{f}.dat", dtype=np.float32).reshape(-1, n)
           for f in ("ux", "uy", "vx", "vy", "sxx", "syy", "sxy")}
    lux = np.fromfile(f"{prefix}_L_ux.dat", dtype=np.float32).reshape(-1, n)
    lvy = np.fromfile(f"{prefix}_L_vy.dat", dtype=np.float32).reshape(-1, n)
    assert out["ux"].shape[0] == nsteps and lux.shape[0] == (nsteps - 1) // 3 + 1
    x = np.fromfile(f"{prefix}_X_x.dat", dtype=np.float32)
    np.testing.assert_array_equal(x, h.side_array(1, 3, "x")[0].astype(np.float32))
    hat_index = {"vx": 0, "vy": 1, "sxx": 2, "sxy": 3, "syy": 4}
    p = GpuDomain(h)
    for step in range(1, nsteps + 1):
        t0 = h.t0 + (step - 1) * h.dt
        U, _ = p.get_side_displacement(1, 3)
        Ub, _ = p.get_side_displacement(1, 2)
        p.time_step_LS(t0, h.dt, final_step=True)
        Fh = p.get_fhat(1, 3)
        np.testing.assert_array_equal(out["ux"][step - 1], U[0].astype(np.float32))
        np.testing.assert_array_equal(out["uy"][step - 1], U[1].astype(np.float32))
        for f, l in hat_index.items():
            np.testing.assert_array_equal(out[f][step - 1], Fh[l].astype(np.float32), err_msg=f)
        if (step - 1) % 3 == 0:
            np.testing.assert_array_equal(lux[(step - 1) // 3], Ub[0].astype(np.float32))
            np.testing.assert_array_equal(lvy[(step - 1) // 3], p.get_fhat(1, 2)[1].astype(np.float32))
        p.time_step_LS(t0, h.dt)
    assert np.abs(lux).max() > 0  # the fault side of the upper block moves


def test_oracle_writer_layout(tmp_path):
    """The oracle's own writer (a restatement of write_output) on the same
    list: item expansion, time windows and strides give the expected sizes."""
    from oracle.binding import OracleDomain
    from oracle.output_writer import OracleOutputs

    text = _problem()
    h = init_domain(text)
    w = OracleOutputs(OracleDomain(h), h, text, tmp_path / "o")
    w.run(1, 30)
    nf = h.iface_n(0)
    size = lambda stem, ext=".dat": (tmp_path / f"o_{stem}{ext}").stat().st_size // 4  # noqa: E731
    assert size("I_V") == 30 * nf and size("I_V", ".t") == 30
    assert size("B_vx") == 8 * h.nx * h.ny  # D%n = 0, 4, ..., 28
    assert size("P_vy") == 30 and size("G_15_V") == 15 and size("G_25_V") == 15
    assert sorted(s for s in w.stems if s.startswith("G_")) == ["G_15_V", "G_25_V", "G_5_V"]


@pytest.mark.gpu
def test_outputs_match_oracle_files(require_gpu, tmp_path):
    """Every file the engine writes against the file the oracle's writer
    writes for the same item: same size and times bit for bit, and float32
    values equal except where the FP64 states, which agree to 1e-10, round
    to neighbouring float32 numbers."""
    from oracle.binding import OracleDomain
    from oracle.output_writer import OracleOutputs

    text = _problem()
    h = init_domain(text)
    g = GpuDomain(h)
    configure_outputs(g, h, text, tmp_path / "g", ring_steps=7)
    g.run(1, 30, nt=h.nt)
    g.output_close()
    w = OracleOutputs(OracleDomain(h), h, text, tmp_path / "o")
    w.run(1, 30)
    assert len(w.stems) == 10  # I: D V S trup, B: vx sxy, P: vy, G: V at nodes 5, 15, 25
    differing = total = 0
    for stem in w.stems:
        for ext in (".t", ".dat"):
            a = (tmp_path / f"g_{stem}{ext}").read_bytes()
            b = (tmp_path / f"o_{stem}{ext}").read_bytes()
            assert len(a) == len(b), f"{stem}{ext}: {len(a)} bytes against the oracle's {len(b)}"
            if ext == ".t":
                assert a == b, f"{stem}.t differs"
                continue
            x, y = np.frombuffer(a, np.float32), np.frombuffer(b, np.float32)
            bad = x != y
            if bad.any():
                tol = 1e-10 * float(np.abs(y).max()) + np.spacing(np.abs(y[bad])).astype(np.float64)
                assert np.all(np.abs(x[bad].astype(np.float64) - y[bad]) <= tol), f"{stem}.dat"
            # values well above round-off of the item's scale are the same float32 numbers
            big = np.abs(y) > 1e-3 * float(np.abs(y).max())
            differing += int((bad & big).sum())
            total += int(big.sum())
    assert differing <= max(4, total // 1000), f"{differing} of {total} float32 values differ"
