"""Checkpoint / resume of the device state in FDMAP's FP64 checkpoint files.

The files follow checkpoint_op (checkpoint.f90:254-288) for a single-process
run: native-endian float64, Fortran column-major arrays, no headers.

  <name>F.ckpt<n>                 F(:,:,l) for l = 1..nF over the global grid,
                                  then DF(:,:,l); with displacement = T, per
                                  component l U(:,:,l) and DU(:,:,l); with
                                  peak = T, pgv and pga; then the perfectly
                                  matched layer fields Wx(:,:,:) and Wy(:,:,:)
                                  when the domain has them (fields.f90:335-429)
  <name>block<b><S>.ckpt<n>       for S = L, R, B, T: per field l the side's
                                  edge values F(:,l), hat variables Fhat(:,l),
                                  prestress F0(:,l); per displacement
                                  component l the boundary displacement U(:,l)
                                  and its rate DU(:,l); then the boundary
                                  energy E(:) and its rate DE(:)
                                                           (fields.f90:432-644)
  <name>iface<i>side<s>.ckpt<n>   for s = 1, 2: the 18 friction fields in
                                  checkpoint_friction order D, Psi, DPsi, trup,
                                  V, O, S, N, S0, N0, Ds, Dn, DDs, DDn, W, DW,
                                  Nreg, DNreg          (friction.f90:491-552)
  <name>.ckpt                     the number of the last checkpoint written

The boundary energies are written as the reference leaves them (E = 0; DE =
1e40, or 0 once a step has run with energy_balance on) and ignored on
reading.  A resume needs F, DF, the boundary displacement and the friction
fields; edge values and hat variables are recomputed in stage 1 of the next
step, exactly as the reference recomputes them after checkpoint_read.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .native import FAULT_FIELDS

SIDES = "LRBT"
COUPLING_FRICTION = 1  # FDMAP_COUPLING_FRICTION


def _edge_values(F: np.ndarray, host, b: int, s: int) -> np.ndarray:
    """Edge row/column of the global fields F (nF, ny, nx) on side s of block b, shape (nF, n)."""
    mgx, pgx, mgy, pgy = host.block_limits(b)
    if s == 0:
        return F[:, mgy - 1:pgy, mgx - 1]
    if s == 1:
        return F[:, mgy - 1:pgy, pgx - 1]
    if s == 2:
        return F[:, mgy - 1, mgx - 1:pgx]
    return F[:, pgy - 1, mgx - 1:pgx]


def checkpoint_write(gpu, host, name: str | Path, number: int) -> list[Path]:
    """Write checkpoint `number` of the device state; returns the files written."""
    name = str(name)
    F, DF = gpu.get_fields(True, True)
    files = []
    p = Path(f"{name}F.ckpt{number}")
    parts = [F.reshape(-1), DF.reshape(-1)]
    if host.displacement:
        U, DU = gpu.get_displacement()
        for l in range(U.shape[0]):
            parts += [U[l].reshape(-1), DU[l].reshape(-1)]
    if host.peak:
        parts += [p.reshape(-1) for p in gpu.get_peak()]
    for w, present in zip(("Wx", "Wy"), host.pml_fields()):
        if present:
            parts.append(gpu.get_pml(w).reshape(-1))
    np.concatenate(parts).astype(np.float64).tofile(p)
    files.append(p)
    for b in range(host.nblocks):
        for s in range(4):
            F0 = host.side_array(b, s, "F0")
            Fh = gpu.get_fhat(b, s)
            Fe = _edge_values(F, host, b, s)
            n = F0.shape[1]
            U, DU = gpu.get_side_displacement(b, s)
            parts = []
            for l in range(host.nF):
                parts += [Fe[l], Fh[l], F0[l]]
            for l in range(U.shape[0]):
                parts += [U[l], DU[l]]
            # boundary energy E and its rate DE: E stays 0 (the reference's boundary flux
            # is a stub); DE keeps its 1e40 start value unless the energy balance is on,
            # where every stage scales it by A (0 in the first stage)
            de = np.zeros(n) if (host.energy_balance and number > 0) else np.full(n, 1e40)
            parts += [np.zeros(n), de]
            p = Path(f"{name}block{b + 1}{SIDES[s]}.ckpt{number}")
            np.concatenate(parts).astype(np.float64).tofile(p)
            files.append(p)
    for i in range(host.nifaces):
        if host.iface_info(i)[3] != COUPLING_FRICTION:  # only frictional interfaces carry state
            continue
        data = np.concatenate([gpu.get_fault(i, f) for f in FAULT_FIELDS]).astype(np.float64)
        for side in (1, 2):
            p = Path(f"{name}iface{i + 1}side{side}.ckpt{number}")
            data.tofile(p)
            files.append(p)
    Path(f"{name}.ckpt").write_text(f"{number}\n")
    return files


def checkpoint_read(gpu, host, name: str | Path, number: int | None = None) -> int:
    """Load checkpoint `number` (default: the last one recorded) into the device
    state; returns the checkpoint number (the step the run resumes after)."""
    name = str(name)
    if number is None:
        number = int(Path(f"{name}.ckpt").read_text().split()[0])
    nn = host.nF * host.ny * host.nx
    a = np.fromfile(f"{name}F.ckpt{number}", dtype=np.float64)
    pml = [w for w, present in zip(("Wx", "Wy"), host.pml_fields()) if present]
    nU = 2 if host.mode == 2 else 1
    plane = host.ny * host.nx
    extra = (2 * nU if host.displacement else 0) + (2 if host.peak else 0)
    if a.size != (2 + len(pml)) * nn + extra * plane:
        raise ValueError(f"{name}F.ckpt{number}: {a.size} values, expected {(2 + len(pml)) * nn + extra * plane}")
    shape = (host.nF, host.ny, host.nx)
    gpu.set_fields(a[:nn].reshape(shape), a[nn:2 * nn].reshape(shape))
    off = 2 * nn
    if host.displacement:
        U = np.stack([a[off + 2 * l * plane:off + (2 * l + 1) * plane] for l in range(nU)])
        DU = np.stack([a[off + (2 * l + 1) * plane:off + (2 * l + 2) * plane] for l in range(nU)])
        gpu.set_displacement(U.reshape(nU, host.ny, host.nx), DU.reshape(nU, host.ny, host.nx))
        off += 2 * nU * plane
    if host.peak:
        gpu.set_peak(a[off:off + plane].reshape(host.ny, host.nx), a[off + plane:off + 2 * plane].reshape(host.ny, host.nx))
        off += 2 * plane
    for k, w in enumerate(pml):
        gpu.set_pml(w, a[off + k * nn:off + (k + 1) * nn].reshape(shape))
    for b in range(host.nblocks):
        for s in range(4):
            mgx, pgx, mgy, pgy = host.block_limits(b)
            n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
            d = np.fromfile(f"{name}block{b + 1}{SIDES[s]}.ckpt{number}", dtype=np.float64)
            if d.size != (3 * host.nF + 2 * nU + 2) * n:
                raise ValueError(f"block {b + 1} side {SIDES[s]} checkpoint: {d.size} values, "
                                 f"expected {(3 * host.nF + 2 * nU + 2) * n}")
            base = 3 * host.nF * n
            U = np.stack([d[base + 2 * l * n:base + (2 * l + 1) * n] for l in range(nU)])
            DU = np.stack([d[base + (2 * l + 1) * n:base + (2 * l + 2) * n] for l in range(nU)])
            gpu.set_side_displacement(b, s, U, DU)
    for i in range(host.nifaces):
        if host.iface_info(i)[3] != COUPLING_FRICTION:
            continue
        n = host.iface_n(i)
        d = np.fromfile(f"{name}iface{i + 1}side1.ckpt{number}", dtype=np.float64)
        if d.size != len(FAULT_FIELDS) * n:
            raise ValueError(f"interface {i + 1} checkpoint: {d.size} values, expected {len(FAULT_FIELDS) * n}")
        for k, f in enumerate(FAULT_FIELDS):
            gpu.set_fault(i, f, d[k * n:(k + 1) * n])
    return number
