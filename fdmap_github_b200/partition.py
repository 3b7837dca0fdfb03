"""Block-aligned partition of one domain over several GPUs.

FDMAP decomposes its domain over MPI processes and, every RK stage, swaps
the interface edge rows between the processes that hold the two sides
(exchange_edge, mpi_routines2d.f90:168-208; called through
exchange_fields_edges, domain.f90:1179-1322).  Here each rank owns whole
blocks (SBP blocks share no grid nodes, so no halo rows cross ranks): it
holds and steps only those blocks, and an interface whose two sides live on
different ranks is solved on both ranks, redundantly and identically, from
its own side's edge values and the peer's, exchanged once per stage.  For
the two-block rupture on two GPUs that is nF x 1601 doubles (77 KB) per
stage and direction.

  plan_partition(host, nranks)   -> PartitionPlan (owner rank of every block,
                                    the interfaces the partition cuts)
  GpuPartition(host, plan, rank) -> this rank's part on its GPU; the edge
                                    exchange is torch.distributed P2P
                                    (NCCL) on the engine's boundary stream
  GpuGroup(parts)                -> all parts driven from one host thread
                                    (fdmap_gpu_group_*: peer copies)
  exchange_edges(...)            -> one round of the exchange for any
                                    backend holding send / receive tensors
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from .domain import GpuDomain, HostDomain, _finish_host
from .native import check_gpu, lib

EXCHANGE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_longlong, C.c_void_p)


@dataclass
class PartitionPlan:
    owner: list[int]                  # rank of every block
    cuts: list[tuple[int, int, int]]  # (interface, rank of its minus side, rank of its plus side)
    nranks: int

    def owned(self, rank: int) -> list[int]:
        return [1 if o == rank else 0 for o in self.owner]

    def pairs(self, rank: int) -> list[tuple[int, int, int]]:
        """(interface, this rank's side 0 = minus / 1 = plus, peer rank) of every cut at `rank`,
        in interface order (the same order on both ranks of a pair)."""
        out = []
        for k, rm, rp in self.cuts:
            if rm == rank:
                out.append((k, 0, rp))
            elif rp == rank:
                out.append((k, 1, rm))
        return out


def plan_partition(host: HostDomain, nranks: int) -> PartitionPlan:
    """Blocks in their input order, cut into `nranks` contiguous runs of
    nearly equal node counts (the reference's decompose1d aligned to block
    starts, mpi_routines.f90:96-221, taken at block granularity)."""
    nb = host.nblocks
    if not 1 <= nranks <= nb:
        raise ValueError(f"{nranks} ranks for {nb} blocks: a block-aligned partition needs 1..{nb} ranks")
    sizes = []
    for b in range(nb):
        mgx, pgx, mgy, pgy = host.block_limits(b)
        sizes.append((pgx - mgx + 1) * (pgy - mgy + 1))
    total = float(sum(sizes))
    # each block goes to the rank whose share of the node count holds the
    # block's centre; if that leaves a rank empty, equal block counts instead
    owner, acc = [], 0.0
    for n in sizes:
        owner.append(min(int((acc + 0.5 * n) / total * nranks), nranks - 1))
        acc += n
    if sorted(set(owner)) != list(range(nranks)):
        owner = [b * nranks // nb for b in range(nb)]
    cuts = []
    for k in range(host.nifaces):
        bm, bp = _iface_blocks(host, k)
        if owner[bm] != owner[bp]:
            cuts.append((k, owner[bm], owner[bp]))
    return PartitionPlan(owner, cuts, nranks)


def _iface_blocks(host: HostDomain, k: int) -> tuple[int, int]:
    """Blocks on the minus and plus side of interface k (fdmap_host_iface_blocks)."""
    out = (C.c_int * 2)()
    rc = host._L.fdmap_host_iface_blocks(host.handle, k, out)
    if rc != 0:
        raise ValueError(f"interface {k}: no block indices ({rc})")
    return int(out[0]), int(out[1])


def exchange_edges(pairs, send, recv, group=None) -> None:
    """One round: for every cut interface, send this rank's edge values to
    the peer and receive the peer's (batched point-to-point, which NCCL runs
    concurrently in one group).  send / recv: tensors in `pairs` order."""
    import torch.distributed as dist

    ops = []
    for (k, side, peer), s, r in zip(pairs, send, recv):
        ops.append(dist.P2POp(dist.isend, s, peer, group))
        ops.append(dist.P2POp(dist.irecv, r, peer, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class _DeviceArray:
    """A device buffer of the engine seen as a CUDA array (no copy)."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False), "version": 3}


class GpuPartition(GpuDomain):
    """This rank's part of the domain on its GPU (fdmap_gpu_create_part).
    With `group` set to a torch.distributed process group (NCCL), the
    exchange callback runs every stage on the engine's boundary stream; a
    GpuGroup drives parts from one thread instead."""

    def __init__(self, host: HostDomain, plan: PartitionPlan, rank: int, device: int = 0, exchange: bool = True,
                 group=None):
        self.host, self.plan, self.rank, self.group = host, plan, rank, group
        self.nx, self.ny, self.nF = host.nx, host.ny, host.nF
        self._owner = None
        self._g = C.c_void_p()
        owned = (C.c_int * host.nblocks)(*plan.owned(rank))
        check_gpu(lib().fdmap_gpu_create_part(host.desc, device, owned, C.byref(self._g)), "fdmap_gpu_create_part")
        _finish_host(host, self)
        self.pairs = plan.pairs(rank)
        self._cb = None
        if exchange and self.pairs:
            self._cb = EXCHANGE_FN(self._exchange)
            check_gpu(lib().fdmap_gpu_set_exchange(self._g, C.cast(self._cb, C.c_void_p), None),
                      "fdmap_gpu_set_exchange")

    def buffers(self, stage: int):
        """(send, receive) device tensors of every cut interface for exchange `stage`."""
        import torch

        send, recv = [], []
        for k, _, _ in self.pairs:
            s, r, n = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.c_longlong()
            check_gpu(lib().fdmap_gpu_part_buffers(self._g, k, stage, C.byref(s), C.byref(r), C.byref(n)),
                      "fdmap_gpu_part_buffers")
            for ptr, dst in ((s, send), (r, recv)):
                addr = C.cast(ptr, C.c_void_p).value
                dst.append(torch.as_tensor(_DeviceArray(addr, n.value), device="cuda"))
        return send, recv

    def _exchange(self, user, stage, stream) -> int:
        try:
            import torch

            with torch.cuda.stream(torch.cuda.ExternalStream(stream)):
                send, recv = self.buffers(stage)
                exchange_edges(self.pairs, send, recv, self.group)
            return 0
        except Exception:  # reported to the engine, which returns an error code
            return 1

    def init_edges(self, t: float | None = None) -> None:
        check_gpu(lib().fdmap_gpu_init_edges(self._g, self.host.t0 if t is None else t), "fdmap_gpu_init_edges")


class GpuGroup:
    """Every part of one domain driven from one host thread: each stage the
    parts pack their edge values, copy their peers' (peer to peer between
    GPUs, or on one GPU), and finish the stage (fdmap_gpu_group_*)."""

    def __init__(self, parts: list[GpuPartition]):
        self.parts = list(parts)
        self._arr = (C.c_void_p * len(self.parts))(*[p._g.value for p in self.parts])
        self.host = self.parts[0].host

    def init_edges(self, t: float | None = None) -> None:
        check_gpu(lib().fdmap_gpu_group_init_edges(self._arr, len(self.parts), self.host.t0 if t is None else t),
                  "fdmap_gpu_group_init_edges")

    def run(self, n_first: int, n_last: int, t_start: float | None = None, dt: float | None = None,
            nt: int | None = None) -> None:
        h = self.host
        check_gpu(lib().fdmap_gpu_group_run(self._arr, len(self.parts), h.t0 if t_start is None else t_start,
                                            h.dt if dt is None else dt, n_first, n_last, h.nt if nt is None else nt),
                  "fdmap_gpu_group_run")

    def synchronize(self) -> None:
        for p in self.parts:
            p.synchronize()
