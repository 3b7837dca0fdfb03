"""Python mirror of FDMAP's host interface for the time-stepping path.

The names follow the reference's Fortran routines:

  init_domain(input_text, base_dir)   -> HostDomain   (domain.f90:45-378 + main.f90:57-116)
  init_domain(..., body_on_device=True)                the O(nx*ny) body left to the device
  GpuDomain(host).time_step_LS(t, dt, final_step)     (time_step.f90:71-167)
  GpuDomain(host).run(n_first, n_last)                (main.f90:168-231 loop body)

Errors raise FdmapError where the reference would call error() / stop.
The arrays returned use FDMAP's global layout F(i, j, l) (Fortran order),
exposed as numpy arrays of shape (nF, ny, nx).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import native
from .native import FAULT_INDEX, check_gpu, check_host, dptr, lib


class HostDomain:
    """An initialised FDMAP domain held in host memory (the Fortran driver's state)."""

    def __init__(self, input_text: str, base_dir: str | Path | None = None, body_on_device: bool = False,
                 native_lib=None):
        # the fdmap_host_* entry points: the engine library, or the same
        # restatement built on its own (a CPU-only caller)
        self._L = native_lib if native_lib is not None else lib()
        self._h = C.c_void_p()
        base = str(base_dir).encode() if base_dir is not None else None
        self.body_on_device = bool(body_on_device)
        flags = native.INIT_BODY_ON_DEVICE if self.body_on_device else 0
        check_host(self._L.fdmap_host_init_ex(input_text.encode(), base, flags, C.byref(self._h)), "init_domain", self._L)
        self._info()

    def _info(self) -> None:
        ints = (C.c_int * 10)()
        dbls = (C.c_double * 5)()
        check_host(self._L.fdmap_host_info(self._h, ints, dbls), "fdmap_host_info", self._L)
        (self.mode, self.nF, self.nx, self.ny, self.nblocks, self.nifaces, self.nt, self.rk_order, self.fd_method,
         het) = list(ints)
        self.heterogeneous = bool(het)
        fl = (C.c_int * 3)()
        check_host(self._L.fdmap_host_body_flags(self._h, fl), "fdmap_host_body_flags", self._L)
        self.displacement, self.peak, self.energy_balance = bool(fl[0]), bool(fl[1]), bool(fl[2])
        (self.t0, self.dt, self.CFL, self.hmin, self.hmax) = list(dbls)

    @property
    def spacing_pending(self) -> bool:
        """True while a domain whose body is left to the device waits for the
        grid spacings (dt, CFL, nt are not known before)."""
        return self.body_on_device and not (self.hmin > 0)

    def set_spacing(self, hmin: float, hmax: float) -> None:
        """Finish set_dt from the grid spacings the device reduced (fdmap_host_set_spacing)."""
        check_host(self._L.fdmap_host_set_spacing(self._h, hmin, hmax), "fdmap_host_set_spacing", self._L)
        self._info()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def desc(self) -> C.c_void_p:
        return C.c_void_p(self._L.fdmap_host_desc(self._h))

    def array(self, name: str) -> np.ndarray:
        """View of a body array ("F", "DF", "x", "y", "xq", ...), shape (k, ny, nx)."""
        n = C.c_longlong()
        p = self._L.fdmap_host_array(self._h, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        a = np.ctypeslib.as_array(p, shape=(n.value,))
        k = n.value // (self.nx * self.ny)
        return a.reshape(k, self.ny, self.nx)

    def iface_n(self, iface: int) -> int:
        n = self._L.fdmap_host_iface_n(self._h, iface)
        if n < 0:
            check_host(n, "fdmap_host_iface_n", self._L)
        return n

    def iface_info(self, iface: int) -> tuple[int, int, int, int]:
        """(direction 0='x' / 1='y', m, p, coupling) of interface `iface`."""
        info = (C.c_int * 4)()
        check_host(self._L.fdmap_host_iface_info(self._h, iface, info), "fdmap_host_iface_info", self._L)
        return tuple(info)

    def iface_xy(self, iface: int) -> tuple[np.ndarray, np.ndarray]:
        n = self.iface_n(iface)
        out = []
        for w in (0, 1):
            p = self._L.fdmap_host_iface_xy(self._h, iface, w)
            out.append(np.ctypeslib.as_array(p, shape=(n,)).copy() if p else np.zeros(n))
        return out[0], out[1]

    def side_array(self, b: int, s: int, name: str) -> np.ndarray:
        """Side array of block b, side s (0..3 = L, R, B, T): "F0" -> (nF, n), "M" -> (5, n), "normal" -> (2, n),
        "x" / "y" -> (1, n)."""
        n = C.c_longlong()
        p = self._L.fdmap_host_side_array(self._h, b, s, name.encode(), C.byref(n))
        if not p:
            raise KeyError(name)
        a = np.ctypeslib.as_array(p, shape=(n.value,)).copy()
        mgx, pgx, mgy, pgy = self.block_limits(b)
        side_n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        return a.reshape(-1, side_n)

    def block_cdiss(self, b: int) -> float:
        """Artificial dissipation coefficient of block b, scaled by CFL/dt (0 = none)."""
        v = self._L.fdmap_host_block_cdiss(self._h, b)
        if v < 0:
            check_host(int(v), "fdmap_host_block_cdiss", self._L)
        return v

    def block_pml(self, b: int) -> dict:
        """pml_list of block b: pmlx, pmly, n, sigma, kappa, mx, px, my, py."""
        fl = (C.c_int * 2)()
        pr = (C.c_double * 7)()
        check_host(self._L.fdmap_host_block_pml(self._h, b, fl, pr), "fdmap_host_block_pml", self._L)
        keys = ("n", "sigma", "kappa", "mx", "px", "my", "py")
        return {"pmlx": bool(fl[0]), "pmly": bool(fl[1]), **dict(zip(keys, list(pr)))}

    def pml_fields(self) -> tuple[bool, bool]:
        """Whether the domain carries Wx and Wy (some block with pmlx / pmly, fields.f90:203-210)."""
        p = [self.block_pml(b) for b in range(self.nblocks)]
        return any(q["pmlx"] for q in p), any(q["pmly"] for q in p)

    def block_limits(self, b: int) -> tuple[int, int, int, int]:
        lim = (C.c_int * 4)()
        check_host(self._L.fdmap_host_block_limits(self._h, b, lim), "fdmap_host_block_limits", self._L)
        return tuple(lim)

    def close(self) -> None:
        if self._h:
            self._L.fdmap_host_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def init_domain(input_text: str, base_dir: str | Path | None = None, body_on_device: bool = False) -> HostDomain:
    """Parse an FDMAP .in text and initialise the domain on the host.  With
    body_on_device the grid, metrics, initial body fields and side impedances
    are built by the engine on the device instead (GpuDomain / GpuEnsemble
    finish the time step from the spacings it reduces)."""
    return HostDomain(input_text, base_dir, body_on_device)


def init_domains(input_texts: list[str], base_dir: str | Path | None = None, threads: int | None = None,
                 body_on_device: bool = False) -> list[HostDomain]:
    """Initialise many independent domains (an ensemble's instances) on a pool
    of host threads; the native initialisation releases the interpreter lock."""
    import os
    from concurrent.futures import ThreadPoolExecutor

    n = threads or min(len(input_texts), os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=max(1, n)) as ex:
        return list(ex.map(lambda t: HostDomain(t, base_dir, body_on_device), input_texts))


class GpuDomain:
    """Device-resident copy of a domain, advanced by the sm_100a kernels."""

    def __init__(self, host: HostDomain, device: int = 0, init_edges: bool = True, _handle=None, _owner=None):
        self.host = host
        self.nx, self.ny, self.nF = host.nx, host.ny, host.nF
        self._owner = _owner  # an instance handle is owned (and freed) by its ensemble
        if _handle is not None:
            self._g = _handle
            return
        self._g = C.c_void_p()
        check_gpu(lib().fdmap_gpu_create(host.desc, device, int(init_edges), C.byref(self._g)), "fdmap_gpu_create")
        _finish_host(host, self)

    def time_params(self) -> tuple[float, float, float, float, float, int]:
        """(t0, dt, CFL, hmin, hmax, nt) as the engine holds them."""
        p = (C.c_double * 5)()
        nt = C.c_int()
        check_gpu(lib().fdmap_gpu_time_params(self._g, p, C.byref(nt)), "fdmap_gpu_time_params")
        return (*list(p), nt.value)

    def get_metric(self, name: str) -> np.ndarray:
        """Metric plane "xq", "xr", "yq", "yr", "Ji" or "J" (dissipative blocks), shape (ny, nx)."""
        out = np.empty((self.ny, self.nx))
        check_gpu(lib().fdmap_gpu_get_metric(self._g, native.METRIC_INDEX[name], dptr(out)), "fdmap_gpu_get_metric")
        return out

    def get_energy(self) -> np.ndarray:
        """Mechanical energy of every block, then their sum, as of the last stage 1 (energy_balance = T)."""
        E = np.empty(self.host.nblocks + 1)
        check_gpu(lib().fdmap_gpu_get_energy(self._g, dptr(E)), "fdmap_gpu_get_energy")
        return E

    def get_displacement(self):
        """Body displacement U and its rate DU (domain_list displacement = T), each (nU, ny, nx)."""
        nU = 2 if self.host.mode == 2 else 1
        U, DU = np.empty((nU, self.ny, self.nx)), np.empty((nU, self.ny, self.nx))
        check_gpu(lib().fdmap_gpu_get_displacement(self._g, dptr(U), dptr(DU)), "fdmap_gpu_get_displacement")
        return U, DU

    def set_displacement(self, U=None, DU=None) -> None:
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        DU = None if DU is None else np.ascontiguousarray(DU, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_displacement(self._g, dptr(U), dptr(DU)), "fdmap_gpu_set_displacement")

    def get_peak(self):
        """Peak ground velocity and acceleration (domain_list peak = T), each (ny, nx)."""
        pgv, pga = np.empty((self.ny, self.nx)), np.empty((self.ny, self.nx))
        check_gpu(lib().fdmap_gpu_get_peak(self._g, dptr(pgv), dptr(pga)), "fdmap_gpu_get_peak")
        return pgv, pga

    def set_peak(self, pgv=None, pga=None) -> None:
        pgv = None if pgv is None else np.ascontiguousarray(pgv, dtype=np.float64)
        pga = None if pga is None else np.ascontiguousarray(pga, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_peak(self._g, dptr(pgv), dptr(pga)), "fdmap_gpu_set_peak")

    def get_side_displacement(self, b: int, s: int):
        """Boundary displacement U and its rate DU of block b, side s: each (nU, n)."""
        mgx, pgx, mgy, pgy = self.host.block_limits(b)
        n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        nU = 2 if self.host.mode == 2 else 1
        U, DU = np.empty(nU * n), np.empty(nU * n)
        check_gpu(lib().fdmap_gpu_get_side_displacement(self._g, b, s, dptr(U), dptr(DU)),
                  "fdmap_gpu_get_side_displacement")
        return U.reshape(nU, n), DU.reshape(nU, n)

    def set_side_displacement(self, b: int, s: int, U=None, DU=None) -> None:
        U = None if U is None else np.ascontiguousarray(U, dtype=np.float64)
        DU = None if DU is None else np.ascontiguousarray(DU, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_side_displacement(self._g, b, s, dptr(U), dptr(DU)),
                  "fdmap_gpu_set_side_displacement")

    def get_pml(self, which: str) -> np.ndarray:
        """Perfectly matched layer field "Wx" or "Wy", shape (nF, ny, nx); zeros outside PML blocks."""
        out = np.empty((self.nF, self.ny, self.nx))
        check_gpu(lib().fdmap_gpu_get_pml(self._g, {"Wx": 0, "Wy": 1}[which], dptr(out)), "fdmap_gpu_get_pml")
        return out

    def set_pml(self, which: str, W) -> None:
        v = np.ascontiguousarray(W, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_pml(self._g, {"Wx": 0, "Wy": 1}[which], dptr(v)), "fdmap_gpu_set_pml")

    def get_side_impedance(self, b: int, s: int) -> np.ndarray:
        """Edge impedances (Zs, Zp, gamma, Ks, Kp) of block b, side s: shape (5, n)."""
        mgx, pgx, mgy, pgy = self.host.block_limits(b)
        n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        out = np.empty(5 * n)
        check_gpu(lib().fdmap_gpu_get_side_impedance(self._g, b, s, dptr(out)), "fdmap_gpu_get_side_impedance")
        return out.reshape(5, n)

    def time_step_LS(self, t0: float, dt: float, final_step: bool = False) -> None:
        check_gpu(lib().fdmap_gpu_time_step(self._g, t0, dt, int(final_step)), "time_step_LS")

    def run(self, n_first: int, n_last: int, t_start: float | None = None, dt: float | None = None,
            nt: int | None = None) -> None:
        h = self.host
        check_gpu(lib().fdmap_gpu_run(self._g, h.t0 if t_start is None else t_start, h.dt if dt is None else dt,
                                      n_first, n_last, h.nt if nt is None else nt), "fdmap_gpu_run")

    def synchronize(self) -> None:
        check_gpu(lib().fdmap_gpu_synchronize(self._g), "fdmap_gpu_synchronize")

    def get_fields(self, want_F: bool = True, want_DF: bool = False):
        F = np.empty((self.nF, self.ny, self.nx)) if want_F else None
        DF = np.empty((self.nF, self.ny, self.nx)) if want_DF else None
        check_gpu(lib().fdmap_gpu_get_fields(self._g, dptr(F), dptr(DF)), "fdmap_gpu_get_fields")
        return F, DF

    def set_fields(self, F=None, DF=None) -> None:
        F = None if F is None else np.ascontiguousarray(F, dtype=np.float64)
        DF = None if DF is None else np.ascontiguousarray(DF, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_fields(self._g, dptr(F), dptr(DF)), "fdmap_gpu_set_fields")

    def get_fault(self, iface: int, field: str) -> np.ndarray:
        out = np.empty(self.host.iface_n(iface))
        check_gpu(lib().fdmap_gpu_get_fault(self._g, iface, FAULT_INDEX[field], dptr(out)), "fdmap_gpu_get_fault")
        return out

    def set_fault(self, iface: int, field: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_set_fault(self._g, iface, FAULT_INDEX[field], dptr(v)), "fdmap_gpu_set_fault")

    def get_fhat(self, b: int, s: int) -> np.ndarray:
        mgx, pgx, mgy, pgy = self.host.block_limits(b)
        n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
        out = np.empty(n * self.nF)
        check_gpu(lib().fdmap_gpu_get_fhat(self._g, b, s, dptr(out)), "fdmap_gpu_get_fhat")
        return out.reshape(self.nF, n)

    # ---- device-side output (fdmap_gpu_output_*)
    def output_add(self, name: str, kind: int, index: int, field: int, mx: int, px: int, sx: int = 1,
                   my: int = 1, py: int = 1, sy: int = 1, nmin: int = 0, nmax: int = 2**62, stride: int = 1) -> None:
        check_gpu(lib().fdmap_gpu_output_add(self._g, name.encode(), kind, index, field, mx, px, sx, my, py, sy,
                                             nmin, nmax, stride), "fdmap_gpu_output_add")

    def output_open(self, prefix: str, ring_steps: int = 512) -> None:
        check_gpu(lib().fdmap_gpu_output_open(self._g, str(prefix).encode(), ring_steps), "fdmap_gpu_output_open")

    def output_flush(self) -> None:
        check_gpu(lib().fdmap_gpu_output_flush(self._g), "fdmap_gpu_output_flush")

    def output_close(self) -> None:
        check_gpu(lib().fdmap_gpu_output_close(self._g), "fdmap_gpu_output_close")

    def fault_max_noalloc(self, iface: int, field: str) -> float:
        """max |field| along interface `iface`, reduced on the device without allocating."""
        out = C.c_double()
        check_gpu(lib().fdmap_gpu_fault_max_noalloc(self._g, iface, FAULT_INDEX[field], C.byref(out)),
                  "fdmap_gpu_fault_max_noalloc")
        return out.value

    def newton_failures(self) -> int:
        """Friction solves whose first Newton attempt failed (the reference's warnings)."""
        return self.newton_counts()[0]

    def newton_counts(self) -> tuple[int, int]:
        """(first-attempt Newton failures, retries that failed too -- where the reference stops)."""
        c = (C.c_longlong * 2)()
        rc = lib().fdmap_gpu_newton_counts(self._g, c)
        if rc not in (0, -4, -5):
            check_gpu(rc, "fdmap_gpu_newton_counts")
        return int(c[0]), int(c[1])

    def status(self) -> int:
        """fdmap_gpu_status: 0, FDMAP_ERR_NEWTON_NOCONV (-4) or FDMAP_ERR_TIMEOUT (-5)."""
        return lib().fdmap_gpu_status(self._g, None)

    def clear_status(self) -> None:
        check_gpu(lib().fdmap_gpu_clear_status(self._g), "fdmap_gpu_clear_status")

    def tile(self) -> tuple[int, int, int]:
        """(tile shape, strip width, rows per row group) of the interior march."""
        t, w, r = C.c_int(), C.c_int(), C.c_int()
        check_gpu(lib().fdmap_gpu_get_tile(self._g, C.byref(t), C.byref(w), C.byref(r)), "fdmap_gpu_get_tile")
        return t.value, w.value, r.value

    def set_tile(self, tile: int) -> None:
        check_gpu(lib().fdmap_gpu_set_tile(self._g, int(tile)), "fdmap_gpu_set_tile")

    @property
    def two_stage(self) -> bool:
        """True when stages run in two-stage interior passes (march_pair.cuh)."""
        r = lib().fdmap_gpu_get_pairs(self._g)
        check_gpu(min(r, 0), "fdmap_gpu_get_pairs")
        return r == 1

    @two_stage.setter
    def two_stage(self, on: bool) -> None:
        check_gpu(lib().fdmap_gpu_set_pairs(self._g, 1 if on else 0), "fdmap_gpu_set_pairs")

    def tune(self, steps: int = 5, dt: float | None = None) -> tuple[int, float]:
        """Autotune the march tile shape; returns (tile, ms per step).  The state is left as it was."""
        t, ms = C.c_int(), C.c_double()
        check_gpu(lib().fdmap_gpu_tune(self._g, self.host.dt if dt is None else dt, steps, C.byref(t), C.byref(ms)),
                  "fdmap_gpu_tune")
        return t.value, ms.value

    def trace(self, capacity: int) -> None:
        """Record one timeline entry per CTA of the stage kernels (0 switches it off)."""
        check_gpu(lib().fdmap_gpu_trace(self._g, int(capacity)), "fdmap_gpu_trace")

    def trace_records(self) -> np.ndarray:
        """(n, 5) int64 array: kind (1 march, 2 closure, 3 interface), SM, CTA, start ns, end ns."""
        n = lib().fdmap_gpu_trace_read(self._g, None, 0)
        if n < 0:
            check_gpu(n, "fdmap_gpu_trace_read")
        buf = (C.c_ulonglong * (3 * max(n, 1)))()
        lib().fdmap_gpu_trace_read(self._g, buf, n)
        a = np.ctypeslib.as_array(buf)[:3 * n].reshape(n, 3).astype(np.int64)
        return np.stack([a[:, 0] & 0xFF, (a[:, 0] >> 8) & 0xFF, a[:, 0] >> 16, a[:, 1], a[:, 2]], axis=1)

    def set_newton_limit(self, imax: int) -> None:
        """Lower the Newton iteration limit (imax = 99 in the reference) to provoke failures."""
        check_gpu(lib().fdmap_gpu_set_newton_limit(self._g, int(imax)), "fdmap_gpu_set_newton_limit")

    def nonfinite_count(self) -> int:
        """Non-finite values in the body fields and the fault V, S, Psi
        (fdmap_gpu_check_finite, which returns FDMAP_ERR_NONFINITE when any)."""
        n = C.c_longlong()
        rc = lib().fdmap_gpu_check_finite(self._g, C.byref(n))
        if rc not in (0, -3):
            check_gpu(rc, "fdmap_gpu_check_finite")
        return n.value

    def launch_count(self) -> int:
        return lib().fdmap_gpu_launch_count(self._g)

    def device_bytes(self) -> int:
        return lib().fdmap_gpu_device_bytes(self._g)

    def close(self) -> None:
        if self._g and self._owner is None:
            lib().fdmap_gpu_destroy(self._g)
        self._g = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _finish_host(host: HostDomain, g: GpuDomain) -> None:
    """A host domain whose body the device built learns its time step from
    the spacings the engine reduced."""
    if host.spacing_pending:
        _, _, _, hmin, hmax, _ = g.time_params()
        host.set_spacing(hmin, hmax)


class GpuEnsemble:
    """Independent domains advanced together by batched launches
    (fdmap_gpu_ensemble_*): one interior march, one interface and one closure
    launch per stage for all instances, one CUDA graph per step."""

    def __init__(self, hosts: list[HostDomain], device: int = 0, init_edges: bool = True):
        self.hosts = list(hosts)
        arr = (C.c_void_p * len(self.hosts))(*[h.desc.value for h in self.hosts])
        self._e = C.c_void_p()
        check_gpu(lib().fdmap_gpu_ensemble_create(arr, len(self.hosts), device, int(init_edges), C.byref(self._e)),
                  "fdmap_gpu_ensemble_create")
        self.instances = []
        for k, h in enumerate(self.hosts):
            g = C.c_void_p()
            check_gpu(lib().fdmap_gpu_ensemble_instance(self._e, k, C.byref(g)), "fdmap_gpu_ensemble_instance")
            self.instances.append(GpuDomain(h, _handle=g, _owner=self))
            _finish_host(h, self.instances[-1])

    def __len__(self) -> int:
        return len(self.hosts)

    def __getitem__(self, k: int) -> GpuDomain:
        return self.instances[k]

    def time_step_LS(self, t0: float, dt: float, final_step: bool = False) -> None:
        check_gpu(lib().fdmap_gpu_ensemble_time_step(self._e, t0, dt, int(final_step)), "ensemble time_step_LS")

    @property
    def dt(self) -> float:
        """Common time step: the smallest of the instances' stable steps."""
        return min(h.dt for h in self.hosts)

    def run(self, n_first: int, n_last: int, t_start: float | None = None, dt: float | None = None,
            nt: int | None = None) -> None:
        h = self.hosts[0]
        check_gpu(lib().fdmap_gpu_ensemble_run(self._e, h.t0 if t_start is None else t_start,
                                               self.dt if dt is None else dt, n_first, n_last,
                                               h.nt if nt is None else nt), "fdmap_gpu_ensemble_run")

    def synchronize(self) -> None:
        check_gpu(lib().fdmap_gpu_ensemble_synchronize(self._e), "fdmap_gpu_ensemble_synchronize")

    @property
    def shape(self) -> tuple[int, int, int]:
        s = (C.c_int * 3)()
        check_gpu(lib().fdmap_gpu_ensemble_get_shape(self._e, s), "fdmap_gpu_ensemble_get_shape")
        return tuple(s)

    @shape.setter
    def shape(self, v) -> None:
        s = (C.c_int * 3)(*v)
        check_gpu(lib().fdmap_gpu_ensemble_set_shape(self._e, s), "fdmap_gpu_ensemble_set_shape")

    def tune(self, steps: int = 5, dt: float | None = None) -> tuple[tuple[int, int, int], float]:
        """Autotune the launch shape; returns (shape, ms per step of the best)."""
        s = (C.c_int * 3)()
        ms = C.c_double()
        check_gpu(lib().fdmap_gpu_ensemble_tune(self._e, self.dt if dt is None else dt, steps, s,
                                                C.byref(ms)), "fdmap_gpu_ensemble_tune")
        return tuple(s), ms.value

    @property
    def tile(self) -> int:
        t = C.c_int()
        check_gpu(lib().fdmap_gpu_ensemble_get_tile(self._e, C.byref(t)), "fdmap_gpu_ensemble_get_tile")
        return t.value

    @tile.setter
    def tile(self, v: int) -> None:
        check_gpu(lib().fdmap_gpu_ensemble_set_tile(self._e, int(v)), "fdmap_gpu_ensemble_set_tile")

    @property
    def two_stage(self) -> bool:
        """True when every instance steps in two-stage interior passes."""
        r = lib().fdmap_gpu_ensemble_get_pairs(self._e)
        check_gpu(min(r, 0), "fdmap_gpu_ensemble_get_pairs")
        return r == 1

    @two_stage.setter
    def two_stage(self, on: bool) -> None:
        check_gpu(lib().fdmap_gpu_ensemble_set_pairs(self._e, 1 if on else 0), "fdmap_gpu_ensemble_set_pairs")

    def launch_count(self) -> int:
        return lib().fdmap_gpu_ensemble_launch_count(self._e)

    def close(self) -> None:
        for g in self.instances:
            g._g = C.c_void_p()
        if self._e:
            lib().fdmap_gpu_ensemble_destroy(self._e)
            self._e = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuAdjoint:
    """Forward/backward pair (fdmap_gpu_adjoint_*): receiver misfit of a
    heterogeneous mode III domain and its gradient with respect to the density
    and shear-modulus fields and, on locked or rate-and-state interfaces, the
    shear prestress of every fault node, by the discrete adjoint with
    checkpoints."""

    def __init__(self, host: HostDomain, receivers, checkpoint_every: int = 45, device: int = 0,
                 store_budget: int = 0):
        self.host = host
        rec = np.asarray(receivers, dtype=np.int32).reshape(-1, 2)  # 1-based (i, j)
        self.nrec = rec.shape[0]
        ri = np.ascontiguousarray(rec[:, 0])
        rj = np.ascontiguousarray(rec[:, 1])
        self._a = C.c_void_p()
        ip = C.POINTER(C.c_int)
        check_gpu(lib().fdmap_gpu_adjoint_create(host.desc, device, self.nrec, ri.ctypes.data_as(ip),
                                                 rj.ctypes.data_as(ip), checkpoint_every, C.byref(self._a)),
                  "fdmap_gpu_adjoint_create")
        if host.spacing_pending:  # body built on the device: the time step follows its spacings
            p = (C.c_double * 5)()
            nt = C.c_int(0)
            check_gpu(lib().fdmap_gpu_adjoint_time_params(self._a, p, C.byref(nt)), "fdmap_gpu_adjoint_time_params")
            host.set_spacing(p[3], p[4])
        if store_budget:
            self.set_store_budget(store_budget)

    def set_store_budget(self, nbytes: int) -> None:
        """Device memory the forward pass with data may keep stage inputs in
        (fdmap_gpu_adjoint_set_store_budget): its last segments stay resident
        and the backward pass reverses them without recomputing; negative =
        all free device memory, 0 = recompute every segment."""
        check_gpu(lib().fdmap_gpu_adjoint_set_store_budget(self._a, int(nbytes)),
                  "fdmap_gpu_adjoint_set_store_budget")

    @property
    def segment_bytes(self) -> int:
        """Bytes of one segment's stage store."""
        return int(lib().fdmap_gpu_adjoint_segment_bytes(self._a))

    @property
    def resident_segments(self) -> int:
        """Segments of the last forward pass with data kept resident."""
        return int(lib().fdmap_gpu_adjoint_resident_segments(self._a))

    def set_material(self, rho: np.ndarray, G: np.ndarray) -> None:
        r = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        g = np.ascontiguousarray(G, dtype=np.float64).reshape(-1)
        check_gpu(lib().fdmap_gpu_adjoint_set_material(self._a, dptr(r), dptr(g)), "fdmap_gpu_adjoint_set_material")

    def forward(self, nt: int | None = None, data: np.ndarray | None = None, dt: float | None = None,
                t_start: float | None = None):
        """Returns (traces[nt, nrec], misfit or None)."""
        h = self.host
        nt = h.nt if nt is None else nt
        tr = np.empty((nt, self.nrec))
        J = C.c_double(0.0)
        d = None if data is None else np.ascontiguousarray(data, dtype=np.float64)
        check_gpu(lib().fdmap_gpu_adjoint_forward(self._a, h.t0 if t_start is None else t_start,
                                                  h.dt if dt is None else dt, nt, dptr(d), dptr(tr), C.byref(J)),
                  "fdmap_gpu_adjoint_forward")
        return tr, (J.value if d is not None else None)

    def backward(self):
        """Returns (dJ/drho, dJ/dG), each shaped (ny, nx)."""
        h = self.host
        gr = np.empty((h.ny, h.nx))
        gg = np.empty((h.ny, h.nx))
        check_gpu(lib().fdmap_gpu_adjoint_backward(self._a, dptr(gr), dptr(gg)), "fdmap_gpu_adjoint_backward")
        return gr, gg

    def fields(self) -> np.ndarray:
        h = self.host
        F = np.empty((h.nF, h.ny, h.nx))
        check_gpu(lib().fdmap_gpu_adjoint_fields(self._a, dptr(F)), "fdmap_gpu_adjoint_fields")
        return F

    @property
    def fault_size(self) -> int:
        """Fault nodes of all interfaces, concatenated in interface order."""
        return int(lib().fdmap_gpu_adjoint_fault_size(self._a))

    def set_prestress(self, S0: np.ndarray) -> None:
        """Background shear stress of every fault node (the stress_file S0 term)."""
        s = np.ascontiguousarray(S0, dtype=np.float64).reshape(-1)
        if s.size != self.fault_size:
            raise ValueError(f"prestress needs {self.fault_size} values, got {s.size}")
        check_gpu(lib().fdmap_gpu_adjoint_set_prestress(self._a, dptr(s)), "fdmap_gpu_adjoint_set_prestress")

    def get_prestress(self) -> np.ndarray:
        s = np.empty(self.fault_size)
        check_gpu(lib().fdmap_gpu_adjoint_get_prestress(self._a, dptr(s)), "fdmap_gpu_adjoint_get_prestress")
        return s

    def prestress_gradient(self) -> np.ndarray:
        """dJ/dS0 per fault node from the last backward pass."""
        g = np.empty(self.fault_size)
        check_gpu(lib().fdmap_gpu_adjoint_prestress_gradient(self._a, dptr(g)),
                  "fdmap_gpu_adjoint_prestress_gradient")
        return g

    def close(self) -> None:
        if self._a:
            lib().fdmap_gpu_adjoint_destroy(self._a)
            self._a = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
