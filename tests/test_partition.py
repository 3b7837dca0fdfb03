"""Block-aligned partition of one domain over ranks (the reference's
exchange_edge between processes, mpi_routines2d.f90:168-208, called from
domain.f90:1179-1322): every rank steps only its blocks and the interface
edge values cross ranks once per stage.

CPU: two gloo ranks run the oracle partitioned (the other rank's block is NaN
on each rank, so any value that does not arrive through the exchange spreads
NaN), and the result equals the single-domain oracle run bit for bit.
GPU: the engine's partitions -- two handles on one GPU driven as a group
(peer copies), and two host threads each driving one handle through the
exchange callback -- equal the single-domain engine run bit for bit."""
from __future__ import annotations

import os
import socket
import threading

import numpy as np
import pytest

from fdmap_github_b200 import FAULT_FIELDS, GpuDomain, init_domain, problems
from fdmap_github_b200.partition import plan_partition

STEPS = 12


def _problems(tmp):
    from tests.test_parity_matrix import fault_text

    return {
        "rupture-II-SW": (problems.rupture_sw(nx=41, ny=21, h=0.5, nt=100), None),
        "rs-III-RAL-het": (problems.heterogeneous_rs_fault(tmp, n=41, h=0.25, nt=100), tmp),
        "x-II-RFL": (fault_text(direction="x", law="RFL", nt=100), None),
        "locked-II": (fault_text(coupling="locked", nt=100), None),
    }


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, tmp, out):
    import torch.distributed as dist

    os.environ["OMP_NUM_THREADS"] = "2"
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        from oracle.binding import OraclePartition

        for name, (text, base) in _problems(tmp).items():
            h = init_domain(text, base)
            plan = plan_partition(h, world)
            part = OraclePartition(h, plan, rank)
            part.run(1, STEPS)
            F = part.get_fields()[0]
            faults = [np.stack([part.get_fault(k, f) for f in FAULT_FIELDS])
                      for k in range(h.nifaces) if h.iface_info(k)[3] == 1]
            np.savez(os.path.join(out, f"{name}_r{rank}.npz"), F=F, owner=np.array(plan.owner), *faults)
    finally:
        dist.destroy_process_group()


def test_plan_partition():
    h = init_domain(problems.rupture_sw(nx=41, ny=21, h=0.5, nt=10))
    p1, p2 = plan_partition(h, 1), plan_partition(h, 2)
    assert p1.owner == [0, 0] and p1.cuts == []
    assert p2.owner == [0, 1] and p2.cuts == [(0, 0, 1)]
    assert p2.pairs(0) == [(0, 0, 1)] and p2.pairs(1) == [(0, 1, 0)]
    with pytest.raises(ValueError):
        plan_partition(h, 3)


def test_two_gloo_ranks_equal_single_domain(tmp_path):
    import torch.multiprocessing as mp

    from oracle.binding import OracleDomain

    out = tmp_path / "out"
    out.mkdir()
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path), str(out)), nprocs=world,
                       start_method="spawn", join=True)
    for name, (text, base) in _problems(str(tmp_path)).items():
        h = init_domain(text, base)
        o = OracleDomain(h)
        o.run(1, STEPS)
        Fo = o.get_fields()[0]
        for r in range(world):
            d = np.load(out / f"{name}_r{r}.npz")
            owner = d["owner"]
            F = d["F"]
            for b in range(h.nblocks):
                mgx, pgx, mgy, pgy = h.block_limits(b)
                blk = (slice(None), slice(mgy - 1, pgy), slice(mgx - 1, pgx))
                if owner[b] == r:
                    assert np.array_equal(F[blk], Fo[blk]), f"{name}: rank {r} block {b} differs"
                else:
                    assert np.isnan(F[blk]).all(), f"{name}: rank {r} computed a block it does not own"
            fr = [k for k in range(h.nifaces) if h.iface_info(k)[3] == 1]
            for q, k in enumerate(fr):
                ref = np.stack([o.get_fault(k, f) for f in FAULT_FIELDS])
                assert np.array_equal(d[f"arr_{q}"], ref), f"{name}: rank {r} fault {k} state differs"
        assert np.abs(Fo).max() > 0


def _gpu_single(text, base):
    h = init_domain(text, base)
    g = GpuDomain(h)
    g.run(1, STEPS)
    F = g.get_fields()[0]
    flt = [np.stack([g.get_fault(k, f) for f in FAULT_FIELDS]) for k in range(h.nifaces) if h.iface_info(k)[3] == 1]
    g.close()
    return h, F, flt


def _check_parts(name, h, F1, flt1, parts):
    for p in parts:
        F = p.get_fields()[0]
        for b in range(h.nblocks):
            if not p.plan.owner[b] == p.rank:
                continue
            mgx, pgx, mgy, pgy = h.block_limits(b)
            blk = (slice(None), slice(mgy - 1, pgy), slice(mgx - 1, pgx))
            assert np.array_equal(F[blk], F1[blk]), f"{name}: partition {p.rank} block {b} differs"
        fr = [k for k in range(h.nifaces) if h.iface_info(k)[3] == 1]
        for q, k in enumerate(fr):
            got = np.stack([p.get_fault(k, f) for f in FAULT_FIELDS])
            assert np.array_equal(got, flt1[q]), f"{name}: partition {p.rank} fault {k} differs"


@pytest.mark.gpu
def test_gpu_group_of_partitions_equals_single_domain(require_gpu, tmp_path):
    from fdmap_github_b200.partition import GpuGroup, GpuPartition

    for name, (text, base) in _problems(tmp_path).items():
        h, F1, flt1 = _gpu_single(text, base)
        plan = plan_partition(h, 2)
        parts = [GpuPartition(h, plan, r, device=0, exchange=False) for r in range(2)]
        grp = GpuGroup(parts)
        grp.init_edges()
        grp.run(1, STEPS)
        grp.synchronize()
        _check_parts(name, h, F1, flt1, parts)
        for p in parts:
            assert p.device_bytes() < 0.75 * GpuDomain(h).device_bytes()  # the peer's body is not held
            p.close()


@pytest.mark.gpu
def test_gpu_partitions_on_two_threads_through_the_callback(require_gpu, tmp_path):
    """Two host threads, one partition each, exchanging through the
    callback: each callback records an event after its own pack, meets the
    other thread on the host, makes its stream wait for the peer's event and
    copies the peer's send buffer into its receive buffer.  No kernel waits
    on another; the ordering is stream and event order."""
    import torch

    from fdmap_github_b200.partition import GpuPartition

    text, base = _problems(tmp_path)["rupture-II-SW"]
    h, F1, flt1 = _gpu_single(text, base)
    plan = plan_partition(h, 2)
    barrier = threading.Barrier(2, timeout=60)
    events = [None, None]
    parts = []

    class ThreadPart(GpuPartition):
        def _exchange(self, user, stage, stream):
            try:
                s = torch.cuda.ExternalStream(stream)
                ev = torch.cuda.Event()
                ev.record(s)
                events[self.rank] = ev
                barrier.wait()  # both packs are queued and their events recorded
                peer = parts[1 - self.rank]
                send_peer, _ = peer.buffers(stage)
                _, recv = self.buffers(stage)
                s.wait_event(events[1 - self.rank])
                with torch.cuda.stream(s):
                    recv[0].copy_(send_peer[0], non_blocking=True)
                barrier.wait()  # both copies are queued before either pack slot is reused
                return 0
            except Exception:
                return 1

    parts.extend(ThreadPart(h, plan, r, device=0) for r in range(2))
    errors = []

    def drive(p):
        try:
            p.init_edges()
            p.run(1, STEPS)
            p.synchronize()
        except Exception as e:  # noqa: BLE001
            errors.append(e)
            barrier.abort()

    th = [threading.Thread(target=drive, args=(p,)) for p in parts]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=120)
    assert not errors, errors
    _check_parts("callback", h, F1, flt1, parts)
    for p in parts:
        p.close()
