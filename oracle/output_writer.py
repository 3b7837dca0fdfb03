"""Output files written from the CPU oracle (TEST INFRASTRUCTURE ONLY).

A restatement of FDMAP's write_output for the oracle's time stepping, used by
tests/ to check the engine's device-side output files against files the oracle
writes itself:

  - the output list grammar of read_output (output.f90:67-294): per item a
    name line, a location line, a line of field names, `tmin tmax stride`,
    then the location's index line (slicex: j; slicey: i; point_body: i j;
    point_iface: k; grid_iface: mx sx px; grid_body / body_grid:
    mx sx px my sy py);
  - the time window of init_output_item (output.f90:414-420):
    nmin = ceiling((tmin - t)/dt), nmax = floor((tmax - t)/dt);
  - write_output_node (output.f90:1011-1074): at step index D%n = n - 1 of
    loop index n, when nmin <= D%n <= nmax and mod(D%n - nmin, stride) == 0,
    append D%t and the values, as float32 (MPI_REAL, mpi_routines.f90:10-13),
    the body fields i fastest;
  - the output point inside stage 1 (time_step.f90:129): the body fields as
    they stand at the step start, the fault fields after the stage-1
    interface solve and rates (the oracle's stage-1 tap).

File names follow the engine's convention: `<prefix>_<name>_<field>.dat` and
`.t`; a grid location expands into one item per point, named by its global
node index(es).  Static fields (x, y) are not written here.
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

BODY = {2: ["vx", "vy", "sxx", "sxy", "syy", "szz"], 3: ["vz", "sxz", "syz"]}
FAULT = ["D", "Psi", "DPsi", "trup", "V", "O", "S", "N", "S0", "N0",
         "Ds", "Dn", "DDs", "DDn", "W", "DW", "Nreg", "DNreg"]


def parse_output_list(text: str) -> list[dict]:
    lines = text.splitlines()
    start = [i for i, ln in enumerate(lines) if ln.strip() == "!---begin:output_list---"]
    if not start:
        return []
    k = start[0] + 1
    items = []
    nidx = {"slicex": 1, "slicey": 1, "point_body": 2, "grid_body": 6, "body_grid": 6}
    while lines[k].strip() != "!---end:output_list---":
        name, loc = lines[k].strip(), lines[k + 1].strip()
        fields = lines[k + 2].split()
        w = lines[k + 3].replace("d", "e").replace("D", "e").split()
        k += 4
        it = {"name": name, "loc": loc, "fields": fields, "tmin": float(w[0]), "tmax": float(w[1]),
              "stride": int(w[2]), "index": []}
        n = nidx.get(loc, 1 if loc.startswith("point_iface") else 3 if loc.startswith("grid_iface") else 0)
        if n:
            it["index"] = [int(v) for v in lines[k].split()[:n]]
            k += 1
        items.append(it)
    return items


class OracleOutputs:
    """Runs an oracle domain step by step and writes the output items."""

    def __init__(self, oracle, host, text: str, prefix: str | Path):
        self.o, self.h, self.prefix = oracle, host, str(prefix)
        self.o.set_tap(True)
        self.files = []  # (file stem, kind, selector, field, nmin, nmax, stride)
        for it in parse_output_list(text):
            nmin = math.ceil((it["tmin"] - host.t0) / host.dt)
            r = (it["tmax"] - host.t0) / host.dt
            nmax = 2 ** 62 if r > 2 ** 62 else math.floor(r)
            for f in it["fields"]:
                if f in ("x", "y"):
                    continue
                for stem, kind, sel in self._expand(it, f):
                    self.files.append((stem, kind, sel, f, nmin, nmax, it["stride"]))
        for stem, *_ in self.files:
            for ext in (".dat", ".t"):
                Path(f"{self.prefix}_{stem}{ext}").write_bytes(b"")

    def _expand(self, it, f):
        loc, name, h = it["loc"], it["name"], self.h
        if "iface" in loc:
            iface = int(loc.split("iface")[1]) - 1
            m = h.iface_info(iface)[1]
            if loc.startswith("point_"):
                return [(f"{name}_{f}", "fault", (iface, [it["index"][0] - m]))]
            if loc.startswith("grid_"):
                a, s, b = it["index"]
                return [(f"{name}_{k}_{f}", "fault", (iface, [k - m])) for k in range(a, b + 1, s)]
            return [(f"{name}_{f}", "fault", (iface, None))]
        if loc == "body":
            box = (1, h.nx, 1, 1, h.ny, 1)
        elif loc.startswith("block"):
            mgx, pgx, mgy, pgy = h.block_limits(int(loc[5:]) - 1)
            box = (mgx, pgx, 1, mgy, pgy, 1)
        elif loc == "point_body":
            i, j = it["index"]
            box = (i, i, 1, j, j, 1)
        elif loc == "slicex":
            box = (1, h.nx, 1, it["index"][0], it["index"][0], 1)
        elif loc == "slicey":
            box = (it["index"][0], it["index"][0], 1, 1, h.ny, 1)
        elif loc == "body_grid":
            mx, sx, px, my, sy, py = it["index"]
            box = (mx, px, sx, my, py, sy)
        elif loc == "grid_body":
            mx, sx, px, my, sy, py = it["index"]
            return [(f"{name}_{i}_{j}_{f}", "body", (i, i, 1, j, j, 1))
                    for j in range(my, py + 1, sy) for i in range(mx, px + 1, sx)]
        else:
            raise ValueError(f"location {loc!r} is not restated here")
        return [(f"{name}_{f}", "body", box)]

    def run(self, n_first: int, n_last: int, nt: int | None = None) -> None:
        h = self.h
        nt = h.nt if nt is None else nt
        for n in range(n_first, n_last + 1):
            t0 = h.t0 + (n - 1) * h.dt
            dn = n - 1
            due = [e for e in self.files if e[4] <= dn <= e[5] and (dn - e[4]) % e[6] == 0]
            F = self.o.get_fields()[0] if any(e[1] == "body" for e in due) else None
            self.o.time_step_LS(t0, h.dt, final_step=(n == nt))
            for stem, kind, sel, f, *_ in due:
                if kind == "body":
                    mx, px, sx, my, py, sy = sel
                    vals = F[BODY[h.mode].index(f), my - 1:py:sy, mx - 1:px:sx]
                else:
                    iface, pts = sel
                    v = self.o.get_fault_tap(iface, f)
                    vals = v if pts is None else v[pts]
                with open(f"{self.prefix}_{stem}.dat", "ab") as fh:
                    np.asarray(vals, dtype=np.float32).tofile(fh)
                with open(f"{self.prefix}_{stem}.t", "ab") as fh:
                    np.asarray([t0], dtype=np.float32).tofile(fh)

    @property
    def stems(self) -> list[str]:
        return [e[0] for e in self.files]
