"""FDMAP's output list on the device-side output of the engine.

`read_output_list(text)` parses the `!---begin:output_list---` section of an
FDMAP input file the way read_output does (output.f90:67-294): per item a
name line, a location line, a line of field names, `tmin tmax stride`, then
the location's index line.  Every field becomes its own item named
`<name>_<field>`; `grid_body` / `grid_iface` expand into point items named
`<name>_<i>_<j>_<field>` / `<name>_<k>_<field>`.

`configure_outputs(gpu, host, text, prefix)` turns those items into
`fdmap_gpu_output_add` calls (time window nmin = ceiling((tmin - t)/dt),
nmax = floor((tmax - t)/dt), output.f90:414-420) and opens the output files
`<prefix>_<name>.dat` / `.t`.  Static fields (x, y, material, which the
reference writes once) are written directly from the host arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from .native import FAULT_INDEX

OUT_FAULT, OUT_BODY, OUT_SIDE, OUT_ENERGY, OUT_SIDE_U = 0, 1, 2, 3, 8
# Ebody / Eblock fields (get_field, domain.f90:517-523, 863-895): Etot, and the
# dissipated energies and rates, zero in the reference (its boundary flux is a stub)
ENERGY_ZERO = {"E", "EL", "ER", "EB", "ET", "DE", "DEL", "DER", "DEB", "DET"}
# body displacement and peak motion (get_field, domain.f90:551-557)
BODY_EXTRA = {"ux": 16, "uz": 16, "uy": 17, "pgv": 24, "pga": 25}
# bndX locations (get_field, domain.f90:763-860): the hat variables by position
# (vx or vz the first, vy the second, sxx, sxy, syy the third to fifth) and the
# boundary displacement; x, y are static
SIDE_HAT = {"vx": 0, "vz": 0, "vy": 1, "sxx": 2, "sxy": 3, "syy": 4}
SIDE_U = {"ux": 0, "uz": 0, "uy": 1}

BODY_FIELDS = {2: ["vx", "vy", "sxx", "sxy", "syy", "szz"], 3: ["vz", "sxz", "syz"]}
STATIC_BODY = {"x", "y", "xq", "xr", "yq", "yr", "J", "rho", "cs", "cp", "G", "M", "gamma", "nu"}
STATIC_FAULT = {"x", "y"}


@dataclass
class OutputItem:
    name: str
    location: str          # body, blockN, ifaceN, point_ifaceN, point_body, body_grid, slicex, slicey, bndXN
    fields: list[str]
    tmin: float
    tmax: float
    stride: int
    index: list[int] = field(default_factory=list)


def read_output_list(text: str) -> list[OutputItem]:
    lines = text.splitlines()
    try:
        k = next(i for i, ln in enumerate(lines) if ln.strip() == "!---begin:output_list---") + 1
    except StopIteration:
        return []
    items: list[OutputItem] = []
    while True:
        name = lines[k].strip()
        if name == "!---end:output_list---":
            return items
        loc = lines[k + 1].strip()
        flds = lines[k + 2].split()
        tt = lines[k + 3].replace("d", "e").replace("D", "e").split()
        tmin, tmax, st = float(tt[0]), float(tt[1]), int(tt[2])
        k += 4
        idx: list[int] = []
        base = loc.split("iface")[0] if "iface" in loc else loc
        if base in ("slicex", "slicey", "point_", "point_body", "grid_", "grid_body", "body_grid"):
            nidx = {"slicex": 1, "slicey": 1, "point_": 1, "point_body": 2, "grid_": 3, "grid_body": 6,
                    "body_grid": 6}[base]
            idx = [int(v) for v in lines[k].split()[:nidx]]
            k += 1
        items.append(OutputItem(name, loc, flds, tmin, tmax, st, idx))


def _window(item: OutputItem, t0: float, dt: float) -> tuple[int, int]:
    nmin = math.ceil((item.tmin - t0) / dt)
    big = 2 ** 62
    r = (item.tmax - t0) / dt
    nmax = big if r > big else math.floor(r)
    return nmin, nmax


def configure_outputs(gpu, host, text: str, prefix: str | Path, ring_steps: int = 512) -> list[str]:
    """Register the input file's output items on `gpu` and open the files.
    Returns the item names registered on the device."""
    mode = host.mode
    names: list[str] = []
    static: list[tuple[str, np.ndarray, int, int]] = []  # name, values, nmin, nmax
    for it in read_output_list(text):
        nmin, nmax = _window(it, host.t0, host.dt)
        loc = it.location
        for f in it.fields:
            nm = f"{it.name}_{f}"
            if "iface" in loc:
                iface = int(loc.split("iface")[1]) - 1
                direction, m, p, _ = host.iface_info(iface)
                n = p - m + 1
                if loc.startswith("point_"):
                    sel = [it.index[0] - m + 1]
                    names_pts = [nm]
                elif loc.startswith("grid_"):
                    a, s, b = it.index[:3]
                    sel = list(range(a - m + 1, b - m + 2, s))
                    names_pts = [f"{it.name}_{m + q - 1}_{f}" for q in sel]
                else:
                    sel = None
                    names_pts = [nm]
                if f in STATIC_FAULT:
                    xy = host.iface_xy(iface)[0 if f == "x" else 1]
                    if sel is None:
                        static.append((nm, xy, nmin, nmax))
                    else:
                        for q, pn in zip(sel, names_pts):
                            static.append((pn, xy[q - 1:q], nmin, nmax))
                    continue
                if f not in FAULT_INDEX:
                    raise ValueError(f"output field {f!r} is not available on interfaces")
                if sel is None:
                    gpu.output_add(nm, OUT_FAULT, iface, FAULT_INDEX[f], 1, n, 1, nmin=nmin, nmax=nmax,
                                   stride=it.stride)
                    names.append(nm)
                else:
                    for q, pn in zip(sel, names_pts):
                        gpu.output_add(pn, OUT_FAULT, iface, FAULT_INDEX[f], q, q, 1, nmin=nmin, nmax=nmax,
                                       stride=it.stride)
                        names.append(pn)
                continue
            if loc == "Ebody" or loc.startswith("Eblock"):
                idx = -1 if loc == "Ebody" else int(loc[6:]) - 1
                if f == "Etot":
                    fld = 0
                elif f in ENERGY_ZERO and loc != "Ebody":
                    fld = 1
                else:
                    raise ValueError(f"output field {f!r} is not available at {loc}")
                gpu.output_add(nm, OUT_ENERGY, idx, fld, 1, 1, 1, nmin=nmin, nmax=nmax, stride=it.stride)
                names.append(nm)
                continue
            if loc.startswith("bnd"):
                # bndXN: side X (L, R, B, T) of block N, every side node
                s = "LRBT".index(loc[3])
                b = int(loc[4:]) - 1
                mgx, pgx, mgy, pgy = host.block_limits(b)
                n = (pgy - mgy + 1) if s < 2 else (pgx - mgx + 1)
                if f in ("x", "y"):
                    static.append((nm, host.side_array(b, s, f)[0], nmin, nmax))
                    continue
                nU = 2 if mode == 2 else 1
                if f in SIDE_U and SIDE_U[f] < nU:
                    fld = OUT_SIDE_U + SIDE_U[f]
                elif f in SIDE_HAT and SIDE_HAT[f] < host.nF:
                    fld = SIDE_HAT[f]
                else:
                    raise ValueError(f"output field {f!r} is not available on block boundaries")
                gpu.output_add(nm, OUT_SIDE, 4 * b + s, fld, 1, n, 1, nmin=nmin, nmax=nmax, stride=it.stride)
                names.append(nm)
                continue
            # body locations: index boxes (mx, px, sx, my, py, sy), global 1-based
            boxes: list[tuple[str, tuple[int, int, int, int, int, int]]] = []
            if loc == "body":
                boxes = [(nm, (1, host.nx, 1, 1, host.ny, 1))]
            elif loc.startswith("block"):
                mgx, pgx, mgy, pgy = host.block_limits(int(loc[5:]) - 1)
                boxes = [(nm, (mgx, pgx, 1, mgy, pgy, 1))]
            elif loc == "point_body":
                i, j = it.index
                boxes = [(nm, (i, i, 1, j, j, 1))]
            elif loc == "grid_body":
                mx, sx, px, my, sy, py = it.index
                boxes = [(f"{it.name}_{i}_{j}_{f}", (i, i, 1, j, j, 1))
                         for j in range(my, py + 1, sy) for i in range(mx, px + 1, sx)]
            elif loc == "body_grid":
                mx, sx, px, my, sy, py = it.index
                boxes = [(nm, (mx, px, sx, my, py, sy))]
            elif loc == "slicex":
                boxes = [(nm, (1, host.nx, 1, it.index[0], it.index[0], 1))]
            elif loc == "slicey":
                boxes = [(nm, (it.index[0], it.index[0], 1, 1, host.ny, 1))]
            else:
                raise ValueError(f"output location {loc!r} is not supported by the device-side output")
            for bn, (mx, px, sx, my, py, sy) in boxes:
                if f in STATIC_BODY:
                    arr = host.array(f)[0]
                    static.append((bn, arr[my - 1:py:sy, mx - 1:px:sx], nmin, nmax))
                    continue
                if f in BODY_FIELDS[mode]:
                    fld = BODY_FIELDS[mode].index(f)
                elif f in BODY_EXTRA and not (mode == 3 and f == "uy"):
                    fld = BODY_EXTRA[f]
                else:
                    raise ValueError(f"output field {f!r} is not a mode {mode} body field")
                gpu.output_add(bn, OUT_BODY, -1, fld, mx, px, sx, my, py, sy,
                               nmin=nmin, nmax=nmax, stride=it.stride)
                names.append(bn)
    # static fields: written once, as the reference does at its first output step
    for nm, vals, nmin, nmax in static:
        if nmin <= 0 <= nmax:
            np.asarray(vals, dtype=np.float32).tofile(f"{prefix}_{nm}.dat")
            np.asarray([host.t0], dtype=np.float32).tofile(f"{prefix}_{nm}.t")
    if names:
        gpu.output_open(str(prefix), ring_steps)
    return names
