"""Batched ensemble: every instance must reproduce its plain single-domain run
bit for bit (same per-node arithmetic, one batched launch per kernel kind),
and the oracle pins one instance."""
from __future__ import annotations

import numpy as np
import pytest

from fdmap_github_b200 import GpuDomain, GpuEnsemble, init_domain, problems
from fdmap_github_b200.native import FAULT_FIELDS
from tests.parity import assert_law_parity


def _instances(tmp_path, sizes, nt=41):
    texts = [problems.ensemble_instance(tmp_path, seed, nx=nx, ny=ny, nt=nt) for seed, (nx, ny) in enumerate(sizes)]
    return [init_domain(t, tmp_path) for t in texts]


def test_von_karman_field_statistics():
    z = problems.von_karman_1d(4001, 0.025, 0.8, 2.0, seed=5)
    assert abs(z.mean()) < 1e-12 and abs(z.std() - 1.0) < 1e-12
    # correlated: neighbouring samples far more alike than independent draws
    assert np.corrcoef(z[:-1], z[1:])[0, 1] > 0.9
    z2 = problems.von_karman_1d(4001, 0.025, 0.8, 2.0, seed=5)
    assert np.array_equal(z, z2)


def test_ensemble_grid_draws():
    grids = [problems.ensemble_grid(s) for s in range(64)]
    assert set(grids) <= set(problems.ENSEMBLE_GRIDS)
    assert len(set(grids)) == 4  # all four sizes occur among 64 seeds


def test_ensemble_instance_init(tmp_path):
    (h,) = _instances(tmp_path, [(81, 41)])
    assert (h.mode, h.nx, h.ny, h.nifaces) == (2, 81, 82, 1)
    S0 = np.fromfile(tmp_path / "stress_0.dat")[:81]
    assert np.all(S0 > 0) and 0.05 < S0.std() / S0.mean() < 0.15


@pytest.mark.gpu
def test_ensemble_matches_plain_runs(require_gpu, tmp_path):
    sizes = [(81, 41), (161, 41), (97, 65)]
    hosts = _instances(tmp_path, sizes)
    ens = GpuEnsemble(hosts)
    dt = ens.dt
    nsteps = 30
    ens.run(1, nsteps, dt=dt)
    ens.synchronize()
    for k, h in enumerate(hosts):
        plain = GpuDomain(h)
        plain.run(1, nsteps, dt=dt)
        Fe, DFe = ens[k].get_fields(True, True)
        Fp, DFp = plain.get_fields(True, True)
        assert np.array_equal(Fe, Fp), f"instance {k}: F differs from the plain run"
        assert np.array_equal(DFe, DFp), f"instance {k}: DF differs from the plain run"
        for f in FAULT_FIELDS:
            assert np.array_equal(ens[k].get_fault(0, f), plain.get_fault(0, f)), f"instance {k}: {f}"
        plain.close()
    ens.close()


@pytest.mark.gpu
def test_ensemble_instance_vs_oracle(require_gpu, tmp_path):
    from oracle.binding import OracleDomain

    hosts = _instances(tmp_path, [(81, 41), (121, 41)])
    ens = GpuEnsemble(hosts)
    dt = ens.dt
    ens.run(1, 25, dt=dt)
    o = OracleDomain(hosts[1])
    o.run(1, 25, dt=dt)
    assert_law_parity(ens[1], o, "RFL", hosts[1], 25, dt=dt)
    ens.close()


@pytest.mark.gpu
def test_ensemble_tuner_and_shapes(require_gpu, tmp_path):
    hosts = _instances(tmp_path, [(81, 41), (161, 81)])
    ens = GpuEnsemble(hosts)
    F0 = [ens[k].get_fields(True, True) for k in range(2)]
    shape, ms = ens.tune(steps=2)
    assert shape[0] in (64, 128, 256) and shape[1] in (32, 64, 128) and shape[2] in (0, 1) and ms > 0
    assert ens.shape == shape
    # tuning leaves the state untouched
    for k in range(2):
        F, DF = ens[k].get_fields(True, True)
        assert np.array_equal(F, F0[k][0]) and np.array_equal(DF, F0[k][1])
    assert ens.tile in (0, 1, 2, 3)
    # every shape and every march tile gives the same answer
    ref = None
    for shp, tile in [((64, 32, 0), 0), ((256, 128, 1), 1), ((128, 64, 1), 2), ((128, 64, 1), 3)]:
        e2 = GpuEnsemble(hosts)
        e2.shape = shp
        e2.tile = tile
        assert e2.tile == tile
        e2.run(1, 12, dt=ens.dt)
        out = [e2[k].get_fields()[0] for k in range(2)]
        if ref is None:
            ref = out
        else:
            for a, b in zip(ref, out):
                assert np.array_equal(a, b)
        e2.close()
    ens.close()


@pytest.mark.gpu
def test_ensemble_two_stage_passes_are_bit_identical(require_gpu, tmp_path):
    """The batched two-stage passes (every instance's stages (1,2), (3,4) in
    one pass) give the bits of the batched stage-by-stage run and of plain
    stage-by-stage runs; the final step issued on top as well."""
    sizes = [(81, 41), (161, 41), (131, 65)]
    hosts = _instances(tmp_path, sizes)
    ens, ens0 = GpuEnsemble(hosts), GpuEnsemble(hosts)
    assert ens.two_stage
    ens0.two_stage = False
    assert not ens0.two_stage
    dt = ens.dt
    for e in (ens, ens0):
        e.run(1, 25, dt=dt)
        e.run(26, 26, dt=dt, nt=26)
        e.synchronize()
    for k, h in enumerate(hosts):
        plain = GpuDomain(h)
        plain.two_stage = False
        plain.run(1, 25, dt=dt)
        plain.run(26, 26, dt=dt, nt=26)
        for other, what in ((ens0[k], "batched stage by stage"), (plain, "plain stage by stage")):
            Fe, DFe = ens[k].get_fields(True, True)
            Fo, DFo = other.get_fields(True, True)
            assert np.array_equal(Fe, Fo) and np.array_equal(DFe, DFo), f"instance {k}: fields differ from the {what} run"
            for f in FAULT_FIELDS:
                assert np.array_equal(ens[k].get_fault(0, f), other.get_fault(0, f)), f"instance {k}: {f} ({what})"
        plain.close()
    ens.close()
    ens0.close()
