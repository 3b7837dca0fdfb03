"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.  It
consumes the same fdmap_desc a HostDomain produces.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import HOST_LIB, LIB, build_oracle

FAULT_FIELDS = ["D", "Psi", "DPsi", "trup", "V", "O", "S", "N", "S0", "N0",
                "Ds", "Dn", "DDs", "DDn", "W", "DW", "Nreg", "DNreg"]

_lib = None


def usable_cpus() -> int:
    """CPUs this process may use: its affinity mask, capped by the cgroup's
    CPU quota (cgroup v2 cpu.max, v1 cfs quota/period), so that OpenMP does
    not run more threads than a container is given time for."""
    n = len(os.sched_getaffinity(0))
    for quota_file, period_file in (("/sys/fs/cgroup/cpu.max", None),
                                    ("/sys/fs/cgroup/cpu/cpu.cfs_quota_us", "/sys/fs/cgroup/cpu/cpu.cfs_period_us")):
        try:
            with open(quota_file) as f:
                parts = f.read().split()
            if period_file is None:
                quota, period = parts[0], parts[1]
            else:
                with open(period_file) as f:
                    quota, period = parts[0], f.read().split()[0]
            if quota not in ("max", "-1") and int(period) > 0:
                n = min(n, max(1, int(quota) // int(period)))
            break
        except (OSError, ValueError, IndexError):
            continue
    return max(1, n)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(str(LIB))
        _DP = C.POINTER(C.c_double)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_void_p]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_init_edges.argtypes = [C.c_void_p, C.c_double]
        L.oracle_time_step.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        L.oracle_run.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
        L.oracle_get_fields.argtypes = [C.c_void_p, _DP, _DP]
        L.oracle_set_fields.argtypes = [C.c_void_p, _DP, _DP]
        L.oracle_get_fault.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.oracle_get_fhat.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.oracle_get_pml.argtypes = [C.c_void_p, C.c_int, _DP]
        L.oracle_get_side_u.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP, _DP]
        L.oracle_get_body_extras.argtypes = [C.c_void_p, _DP, _DP, _DP, _DP]
        L.oracle_get_energy.argtypes = [C.c_void_p, _DP]
        L.oracle_newton_failures.restype = C.c_longlong
        L.oracle_newton_failures.argtypes = [C.c_void_p]
        L.oracle_newton_stops.restype = C.c_longlong
        L.oracle_newton_stops.argtypes = [C.c_void_p]
        L.oracle_set_newton_limit.argtypes = [C.c_void_p, C.c_int]
        L.oracle_set_newton_tolerance.argtypes = [C.c_void_p, C.c_double]
        L.oracle_num_threads.restype = C.c_int
        L.oracle_set_num_threads.argtypes = [C.c_int]
        if "OMP_NUM_THREADS" not in os.environ:
            L.oracle_set_num_threads(min(L.oracle_num_threads(), usable_cpus()))
        L.oracle_set_tap.argtypes = [C.c_void_p, C.c_int]
        L.oracle_get_fault_tap.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.oracle_set_fault.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.oracle_set_side_u.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP, _DP]
        L.oracle_set_body_extras.argtypes = [C.c_void_p, _DP, _DP, _DP, _DP]
        L.oracle_set_pml.argtypes = [C.c_void_p, C.c_int, _DP]
        L.oracle_set_owned.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.oracle_set_exchange.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.oracle_get_iface_edge.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        L.oracle_set_iface_edge.argtypes = [C.c_void_p, C.c_int, C.c_int, _DP]
        _lib = L
    return _lib


_host_lib = None


def host_lib() -> C.CDLL:
    """The host initialisation (fdmap_host_*) built on its own into
    oracle/_build/libhost_init.so: the CPU arm's init_domain, which loads no
    library of the GPU package."""
    global _host_lib
    if _host_lib is None:
        build_oracle()
        from fdmap_github_b200.native import SIGNATURES

        L = C.CDLL(str(HOST_LIB))
        for name, (res, args) in SIGNATURES.items():
            if name.startswith("fdmap_host_"):
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
        _host_lib = L
    return _host_lib


def init_domain_cpu(input_text: str, base_dir=None):
    """init_domain through libhost_init.so (same restatement, same descriptor)."""
    from fdmap_github_b200.domain import HostDomain

    return HostDomain(input_text, base_dir, native_lib=host_lib())


def _p(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


class OracleDomain:
    """CPU restatement of FDMAP's time stepping on a copy of a HostDomain."""

    def __init__(self, host, init_edges: bool = True):
        self.host = host
        self.nx, self.ny, self.nF = host.nx, host.ny, host.nF
        self._o = lib().oracle_create(host.desc)
        if not self._o:
            raise RuntimeError("oracle_create rejected the descriptor")
        if init_edges:
            lib().oracle_init_edges(self._o, host.t0)

    def time_step_LS(self, t0: float, dt: float, final_step: bool = False) -> None:
        if lib().oracle_time_step(self._o, t0, dt, int(final_step)) != 0:
            raise RuntimeError("oracle_time_step failed")

    def run(self, n_first: int, n_last: int, t_start=None, dt=None, nt=None) -> None:
        h = self.host
        if lib().oracle_run(self._o, h.t0 if t_start is None else t_start, h.dt if dt is None else dt,
                            n_first, n_last, h.nt if nt is None else nt) != 0:
            raise RuntimeError("oracle_run failed")

    def get_fields(self, want_F: bool = True, want_DF: bool = False):
        F = np.empty((self.nF, self.ny, self.nx)) if want_F else None
        DF = np.empty((self.nF, self.ny, self.nx)) if want_DF else None
        lib().oracle_get_fields(self._o, _p(F), _p(DF))
        return F, DF

    def set_fields(self, F=None, DF=None) -> None:
        F = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        DF = None if DF is None else np.ascontiguousarray(DF, dtype=np.float64)
        lib().oracle_set_fields(self._o, _p(F), _p(DF))

    def get_fault(self, iface: int, field: str) -> np.ndarray:
        out = np.empty(self.host.iface_n(iface))
        rc = lib().oracle_get_fault(self._o, iface, FAULT_FIELDS.index(field), _p(out))
        if rc != 0:
            raise RuntimeError(f"oracle_get_fault failed ({rc})")
        return out

    def set_fault(self, iface: int, field: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        if lib().oracle_set_fault(self._o, iface, FAULT_FIELDS.index(field), _p(v)) != 0:
            raise RuntimeError("oracle_set_fault failed")

    def set_tap(self, on: bool = True) -> None:
        """Keep each step's stage-1 fault fields (the reference's output point)."""
        lib().oracle_set_tap(self._o, int(on))

    def get_fault_tap(self, iface: int, field: str) -> np.ndarray:
        out = np.empty(self.host.iface_n(iface))
        if lib().oracle_get_fault_tap(self._o, iface, FAULT_FIELDS.index(field), _p(out)) != 0:
            raise RuntimeError("no stage-1 fault fields kept (set_tap first)")
        return out

    def set_side_displacement(self, b: int, s: int, U=None, DU=None) -> None:
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        DU = None if DU is None else np.ascontiguousarray(DU, dtype=np.float64)
        lib().oracle_set_side_u(self._o, b, s, _p(U), _p(DU))

    def set_displacement(self, U=None, DU=None) -> None:
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        DU = None if DU is None else np.ascontiguousarray(DU, dtype=np.float64)
        if lib().oracle_set_body_extras(self._o, _p(U), _p(DU), None, None):
            raise RuntimeError("the domain does not track the body displacement")

    def set_peak(self, pgv=None, pga=None) -> None:
        pgv = None if pgv is None else np.ascontiguousarray(pgv, dtype=np.float64)
        pga = None if pga is None else np.ascontiguousarray(pga, dtype=np.float64)
        if lib().oracle_set_body_extras(self._o, None, None, _p(pgv), _p(pga)):
            raise RuntimeError("the domain does not track peak motion")

    def set_pml(self, which: str, W) -> None:
        v = np.ascontiguousarray(W, dtype=np.float64)
        if lib().oracle_set_pml(self._o, {"Wx": 0, "Wy": 1}[which], _p(v)):
            raise RuntimeError("the domain has no such PML field")

    def get_fhat(self, b: int, s: int) -> np.ndarray:
        mgx, pgx, mgy, pgy = self.host.block_limits(b)
        n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        out = np.empty(n * self.nF)
        lib().oracle_get_fhat(self._o, b, s, _p(out))
        return out.reshape(self.nF, n)

    def get_displacement(self):
        """Body displacement U and its rate DU, each (nU, ny, nx)."""
        nU = 2 if self.host.mode == 2 else 1
        U, DU = np.empty((nU, self.ny, self.nx)), np.empty((nU, self.ny, self.nx))
        if lib().oracle_get_body_extras(self._o, _p(U), _p(DU), None, None):
            raise RuntimeError("the domain does not track the body displacement")
        return U, DU

    def get_energy(self) -> np.ndarray:
        """Mechanical energy of every block, then their sum (energy_balance = T)."""
        E = np.empty(self.host.nblocks + 1)
        if lib().oracle_get_energy(self._o, _p(E)):
            raise RuntimeError("the domain does not track the energy")
        return E

    def get_peak(self):
        """Peak ground velocity and acceleration, each (ny, nx)."""
        pgv, pga = np.empty((self.ny, self.nx)), np.empty((self.ny, self.nx))
        if lib().oracle_get_body_extras(self._o, None, None, _p(pgv), _p(pga)):
            raise RuntimeError("the domain does not track peak motion")
        return pgv, pga

    def get_side_u(self, b: int, s: int):
        """Boundary displacement U and its rate DU of block b, side s: each (nU, n)."""
        mgx, pgx, mgy, pgy = self.host.block_limits(b)
        n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        nU = 2 if self.host.mode == 2 else 1
        U, DU = np.empty(n * nU), np.empty(n * nU)
        lib().oracle_get_side_u(self._o, b, s, _p(U), _p(DU))
        return U.reshape(nU, n), DU.reshape(nU, n)

    def get_side_displacement(self, b: int, s: int):
        """As get_side_u (the name GpuDomain uses)."""
        return self.get_side_u(b, s)

    def get_pml(self, which: str) -> np.ndarray:
        """PML field "Wx" or "Wy", shape (nF, ny, nx); zeros where the domain has none."""
        out = np.empty((self.nF, self.ny, self.nx))
        lib().oracle_get_pml(self._o, {"Wx": 0, "Wy": 1}[which], _p(out))
        return out

    def newton_failures(self) -> int:
        return lib().oracle_newton_failures(self._o)

    def newton_counts(self) -> tuple[int, int]:
        """(first-attempt Newton failures, retries that failed too)."""
        return lib().oracle_newton_failures(self._o), lib().oracle_newton_stops(self._o)

    def set_newton_tolerance(self, scale: float) -> None:
        """Newton residual tolerance = scale x the reference's atolR."""
        if lib().oracle_set_newton_tolerance(self._o, float(scale)) != 0:
            raise ValueError("bad tolerance scale")

    def set_newton_limit(self, imax: int) -> None:
        if lib().oracle_set_newton_limit(self._o, int(imax)) != 0:
            raise ValueError("bad Newton iteration limit")

    def close(self) -> None:
        if self._o:
            lib().oracle_destroy(self._o)
            self._o = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def num_threads() -> int:
    return lib().oracle_num_threads()


ORACLE_EXCHANGE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_longlong)


class OraclePartition(OracleDomain):
    """One rank's part of a block-aligned partition on the CPU oracle: the
    other ranks' blocks are NaN here, and every stage the interface edge
    values are exchanged with the peers through torch.distributed (gloo),
    by the same exchange_edges the GPU partitions use."""

    def __init__(self, host, plan, rank: int, group=None):
        super().__init__(host, init_edges=False)
        self.plan, self.rank, self.group = plan, rank, group
        owned = (C.c_int * host.nblocks)(*plan.owned(rank))
        lib().oracle_set_owned(self._o, owned)
        self.pairs = plan.pairs(rank)
        self.errors = []
        self._cb = ORACLE_EXCHANGE(self._exchange)
        lib().oracle_set_exchange(self._o, C.cast(self._cb, C.c_void_p), None)
        if lib().oracle_init_edges(self._o, host.t0) != 0:
            raise RuntimeError("initial edge exchange failed: " + "; ".join(self.errors))

    def _exchange(self, user, stage) -> int:
        try:
            import torch

            from fdmap_github_b200.partition import exchange_edges

            send, recv = [], []
            for k, side, _ in self.pairs:
                n = self.host.iface_n(k)
                buf = np.empty(self.nF * n)
                lib().oracle_get_iface_edge(self._o, k, side, _p(buf))
                send.append(torch.from_numpy(buf))
                recv.append(torch.empty(self.nF * n, dtype=torch.float64))
            exchange_edges(self.pairs, send, recv, self.group)
            for (k, side, _), r in zip(self.pairs, recv):
                v = np.ascontiguousarray(r.numpy())
                lib().oracle_set_iface_edge(self._o, k, 1 - side, _p(v))
            return 0
        except Exception as e:  # noqa: BLE001  (reported as a failed step)
            self.errors.append(repr(e))
            return 1

