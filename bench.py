#!/usr/bin/env python
"""Benchmark of the FDMAP time-stepping hot path on B200.

Workload (default "rupture"): mode II dynamic rupture, two blocks of
1601 x 801 nodes (dx = 25 m) joined at a planar slip-weakening fault, LS-RK4
at CFL 0.5 -- the configuration the headline metric is quoted on.  A step is
one full low-storage RK4 time step (5 stages) over all 2,564,802 nodes.

  value   FP64 node-updates/s of the whole job (all ranks), device-resident state,
          K steps timed with CUDA events on the engine's stream
  e2e     the same metric through the public C ABI with host buffers: the
          initial state upload, the fault output of every step (slip, slip
          rate, shear stress, rupture time as float32 time series, gathered
          on the device and written to files) and the final field download
          are inside the timed region
  roofline  the fused stencil kernel's achieved HBM bandwidth (algorithmic
          bytes per launch / its mean CUDA-event duration) against the measured
          copy bandwidth

Multi-GPU: one replica per rank (weak scaling), no data-path collective.
`--impl reference` times the CPU restatement of the reference (the Fortran/MPI
reference cannot be built in this image) on the host cores, on the same
workload, steps and warm-up; both arms print the same `config`.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from fdmap_github_b200 import FdmapError, GpuDomain, init_domain, problems  # noqa: E402
from fdmap_github_b200.native import FAULT_INDEX  # noqa: E402

METRIC = "FP64 node-updates/s"
UNIT = "node-updates/s"

# Algorithmic HBM bytes per node per RK stage of the fused stencil kernel
# (compulsory reads and writes of one stage):
#   mode II: F 6 read + 6 write, DF 5 read + 6 write, metrics xq,xr,yq,yr,Ji 5 read
#   mode III: F 3+3, DF 3+3, metrics 5;  heterogeneous adds rho,G (III) / 5 arrays (II)
# A stage whose RK coefficient A is 0 (the first) does not read DF: NR_DF
# fewer doubles per node (DF6 is never read: rates_szz overwrites it).
BYTES_PER_NODE_STAGE = {(2, False): 28 * 8, (2, True): 33 * 8, (3, False): 17 * 8, (3, True): 19 * 8}
NR_DF = {2: 5, 3: 3}
RK_STAGES = {1: 1, 2: 2, 3: 3, 4: 5}


def extra_bytes_per_node_stage(host) -> tuple[int, int]:
    """(bytes in every stage, bytes not read in stage 1) a node moves for the
    domain's extras: the Jacobian of dissipative blocks (1 read); per PML
    layer W read + written and DW read + written (nF planes each, DW unread
    when A = 0) and the two damping planes; body displacement U, DU (nU
    planes each, read + written; DU unread when A = 0)."""
    nF, every, first_skip = host.nF, 0, 0
    if any(host.block_cdiss(b) > 0 for b in range(host.nblocks)):
        every += 8
    px, py = host.pml_fields()
    if px or py:
        every += 2 * 8
        for on in (px, py):
            if on:
                every += 4 * nF * 8
                first_skip += nF * 8
    if host.displacement:
        nU = 2 if host.mode == 2 else 1
        every += 4 * nU * 8
        first_skip += nU * 8
    return every, first_skip


PI_OF = {2: 1, 4: 2, 6: 3}
NBST_OF = {2: 1, 4: 4, 6: 6}


def nodes_at_least(host, k: int) -> int:
    """Nodes at distance >= k from their block's nearest edge, summed over blocks."""
    n = 0
    for b in range(host.nblocks):
        mgx, pgx, mgy, pgy = host.block_limits(b)
        nx, ny = pgx - mgx + 1, pgy - mgy + 1
        n += max(nx - 2 * k, 0) * max(ny - 2 * k, 0)
    return n


def pair_bytes(host, reads_rates: bool) -> int:
    """Algorithmic bytes of one two-stage interior pass (march_pair.cuh): at
    every interior node (distance >= nbst from the edges) the stage input is
    read once -- the NR rate fields, szz (mode II), the five metric planes and,
    when the first stage's A is not 0, the NR input rates; at nodes >= nbst + PI
    the pass writes the second stage's fields and rates (2 NF planes); nearer
    the edges it writes the first stage's fields (nbst .. nbst + 2 PI) and
    rates (nbst .. nbst + PI) for the band kernel."""
    nr, nf = (5, 6) if host.mode == 2 else (3, 3)
    nbst, pi = NBST_OF[host.fd_method], PI_OF[host.fd_method]
    n_int = nodes_at_least(host, nbst)
    reads = n_int * (nr + (1 if host.mode == 2 else 0) + 5 + (nr if reads_rates else 0))
    writes = (nodes_at_least(host, nbst + pi) * 2 * nf
              + (n_int - nodes_at_least(host, nbst + 2 * pi)) * nf
              + (n_int - nodes_at_least(host, nbst + pi)) * nf)
    return 8 * (reads + writes)


def bytes_per_node_update(mode: int, het: bool, rk_order: int, host=None) -> int:
    """Algorithmic bytes of one node over one full step (all stages; DF unread in stage 1)."""
    ex, skip = extra_bytes_per_node_stage(host) if host is not None else (0, 0)
    return RK_STAGES[rk_order] * (BYTES_PER_NODE_STAGE[(mode, het)] + ex) - NR_DF[mode] * 8 - skip


def shared_config(info: dict, host) -> dict:
    """The workload as both arms report it (identical dicts): shapes, step
    count of the full run, and how the inputs relate to the 126 MB L2."""
    state = host.nx * host.ny * (2 * host.nF + 5) * 8  # F, DF and the five metric planes
    l2 = (f"inputs larger than L2 (state {state / 1e9:.2f} GB > 126 MB), no flush needed" if state > 126e6
          else f"state {state / 1e6:.1f} MB fits in L2: latency bound, roofline fraction not meaningful")
    return {**info, "rk_stages_per_step": RK_STAGES[host.rk_order], "nt_reference": host.nt, "l2": l2}


def workload(name: str, tmpdir: Path):
    if name == "rupture":
        return problems.rupture_sw(), None, {"workload": "mode II slip-weakening rupture, 2 blocks x 1601x801, dx 25 m, LS-RK4 CFL 0.5",
                                             "nodes": 1601 * 1602, "fault_nodes": 1601}
    if name == "pulse":
        return problems.antiplane_pulse(), None, {"workload": "mode III SH pulse, 1 block 201x201, LS-RK4 CFL 0.5", "nodes": 201 * 201}
    if name == "roughfault":
        text = problems.rough_fault_rs(tmpdir)
        return text, tmpdir, {"workload": "mode II rate-and-state (RFL) rough fault, 2 curvilinear blocks x 2001x1001",
                              "nodes": 2001 * 2002, "fault_nodes": 2001}
    if name == "rupture_cdiss":
        return problems.rupture_sw(cdiss=0.3), None, {
            "workload": "mode II slip-weakening rupture, 2 blocks x 1601x801, dx 25 m, artificial dissipation "
                        "Cdiss 0.3, LS-RK4 CFL 0.5", "nodes": 1601 * 1602, "fault_nodes": 1601}
    if name == "pml":
        return problems.pml_pulse(n=2001, L=40.0, width=3.0, nt=4001), None, {
            "workload": "mode II P-SV pulse, 1 block 2001x2001 (dx 20 m) with a 3 km perfectly matched layer "
                        "(Wx and Wy on every node), LS-RK4 CFL 0.5", "nodes": 2001 * 2001}
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """Samples SM clocks and clock-event (throttle) reasons through NVML every
    few milliseconds while the timed region runs (read-only queries)."""

    PERIOD_S = 0.005
    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple[int, int]] = []
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._sample()
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        except Exception:
            self._t = None
        return self

    def _sample(self):
        nv = self._nv
        mhz = nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM)
        try:
            rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self._h)
        except AttributeError:
            rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
        self.samples.append((mhz, rs))

    def _run(self):
        while not self._stop.wait(self.PERIOD_S):
            try:
                self._sample()
            except Exception:
                return

    def __exit__(self, *exc):
        if self._t is not None:
            self._stop.set()
            self._t.join(timeout=5)
            try:
                self._sample()
            except Exception:
                pass

    def summary(self) -> dict:
        sm = [m for m, _ in self.samples]
        reasons = set()
        for _, rs in self.samples:
            for name, bit in self.REASONS.items():
                if rs & bit:
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvml"}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(config_key: str, kernel: str = "march_kernel"):
    """DRAM bytes per launch of `kernel` from the committed ncu summaries, if any."""
    for p in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(rf"traffic_bytes_per_launch\[{config_key}:{kernel}\]\s*=\s*([0-9.eE+]+)", p.read_text())
        if m:
            return float(m.group(1))
    return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return world, rank, local


def barrier_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_gpu(args) -> None:
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    tmp = Path(tempfile.mkdtemp(prefix=f"fdmap_bench_r{rank}_"))
    text, base, info = workload(args.workload, tmp)
    host = init_domain(text, base)
    nodes = host.nx * host.ny
    het = host.heterogeneous
    # a dedicated stream: the engine's kernels and the timing events share it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    # ---- device-resident throughput (value)
    g = GpuDomain(host, device=local)
    lib_set_stream(g, stream)
    nt_inf = 1 << 30
    # the autotuner picks the march tile (the state is left as it was)
    try:
        tile, tune_ms = g.tune(steps=3)
        tile_info = dict(zip(("tile", "strip_width", "rows_per_group"), g.tile()), tuned_ms_per_step=tune_ms)
    except FdmapError:
        tile, tile_info = None, {"tile": None, "kernel": "tiled interior kernel"}
    g.run(1, args.warmup, nt=nt_inf)
    g.synchronize()
    barrier(world)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        barrier(world)
        start.record(stream)
        g.run(args.warmup + 1, args.warmup + args.steps, nt=nt_inf)
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    ms_max = barrier_max(ms, world)
    launches = g.launch_count()
    value = world * nodes * args.steps / (ms_max * 1e-3)

    # ---- per-kernel durations for the roofline (same kernels, event-bracketed)
    from fdmap_github_b200.native import lib
    import ctypes as C

    lib().fdmap_gpu_profile(g._g, 1)
    g.run(args.warmup + args.steps + 1, args.warmup + 2 * args.steps, nt=nt_inf)
    kms = (C.c_double * 5)()
    kn = (C.c_longlong * 5)()
    lib().fdmap_gpu_profile_read_kinds(g._g, 5, kms, kn)
    lib().fdmap_gpu_profile(g._g, 0)
    stencil_ms = kms[0] / max(kn[0], 1)
    closure_ms = kms[1] / max(kn[1], 1)
    edge_ms = kms[2] / max(kn[2], 1)
    pair_ms = kms[3] / max(kn[3], 1)
    band_ms = kms[4] / max(kn[4], 1)
    prof_kinds = {k: {"launches": int(kn[i]), "mean_ms": kms[i] / max(kn[i], 1)}
                  for i, k in enumerate(("march", "closure", "interface", "pair_march", "band")) if kn[i]}
    pairs = bool(g.two_stage)
    nst = RK_STAGES[host.rk_order]
    bps = BYTES_PER_NODE_STAGE[(host.mode, het)]
    n_int = interior_nodes(host)
    # mean algorithmic bytes of one interior-kernel launch over the step's
    # stages: every stage reads F, metrics and DF, except stage 1 (A = 0)
    ex, skip = extra_bytes_per_node_stage(host)
    stage_bytes = [n_int * (bps + ex - ((NR_DF[host.mode] * 8 + skip) if q == 0 else 0)) for q in range(nst)]
    alg_bytes = sum(stage_bytes) / nst
    peaks = measured_peaks()
    # stage by stage, every stage moves the whole state (stage_bytes); with
    # two-stage passes, stages (1,2) and (3,4) are one pass each and only the
    # last stage of an odd count runs alone
    npairs = nst // 2 if pairs else 0
    pass_bytes = [pair_bytes(host, q > 0) for q in range(npairs)]
    single_bytes = stage_bytes[2 * npairs:]
    if pairs:
        kernel, mean_ms = "march_pair_kernel", pair_ms
        launch_bytes = sum(pass_bytes) / npairs
    else:
        kernel, mean_ms = "march_kernel", stencil_ms
        launch_bytes = alg_bytes
    achieved = launch_bytes / (mean_ms * 1e-3) / 1e9
    march_bytes = (sum(single_bytes) / len(single_bytes)) if single_bytes else alg_bytes
    march_gbs = march_bytes / (stencil_ms * 1e-3) / 1e9 if kn[0] else None
    # the whole step against the same peak: the schedule's own algorithmic
    # bytes (interior passes and stages, plus the closure strips' stage-by-
    # stage bytes), and the stage-by-stage bytes of every node (the work the
    # step does, counted as one pass per stage)
    n_edge = nodes - n_int
    sched_bytes = sum(pass_bytes) + sum(single_bytes) + n_edge * bytes_per_node_update(host.mode, het,
                                                                                      host.rk_order, host)
    step_s = ms_max / args.steps * 1e-3
    step_bytes = nodes * bytes_per_node_update(host.mode, het, host.rk_order, host)
    step_gbs = sched_bytes / step_s / 1e9
    unfused_gbs = step_bytes / step_s / 1e9
    survey_bytes = nodes * RK_STAGES[host.rk_order] * (BYTES_PER_NODE_STAGE[(host.mode, het)] - 5 * 8)
    newton_fail = g.newton_failures()
    g.close()

    # ---- end to end through the public API with host buffers: every timed
    # repetition starts a fresh run from the initial state held in pinned
    # host memory (fields and the 18 fault fields uploaded), runs the steps
    # with the fault time series written through the device-side output, and
    # reads the final fields back into pinned memory.  DF is not uploaded:
    # the first stage multiplies it by A(1) = 0 and never reads it.
    g2 = GpuDomain(host, device=local, init_edges=False)
    lib_set_stream(g2, stream)
    if tile is not None:
        g2.set_tile(tile)
    if g2.two_stage != pairs:
        g2.two_stage = pairs  # the tuner's choice for the first handle
    nf = info.get("fault_nodes", 0)
    # the fault registers as the descriptor gives them, before the initial edge solve
    fault0 = {f: torch.from_numpy(g2.get_fault(0, f)).pin_memory().numpy() for f in FAULT_INDEX} if nf else {}
    lib().fdmap_gpu_init_edges(g2._g, host.t0)
    g2.run(1, args.warmup, nt=nt_inf)  # captures the step graphs (set-up, untimed)
    g2.synchronize()
    F0 = np.ascontiguousarray(host.array("F"))
    pin_F = torch.from_numpy(F0).pin_memory()
    pin_out = torch.empty(F0.shape, dtype=torch.float64).pin_memory()  # the run's result, read back
    out_dir = Path(tempfile.mkdtemp(prefix=f"fdmap_bench_out_r{rank}_"))
    if nf:
        for f in ("D", "V", "S", "trup"):
            g2.output_add(f"fault_{f}", 0, 0, FAULT_INDEX[f], 1, nf, 1, nmin=0, nmax=1 << 62, stride=1)
        g2.output_open(str(out_dir / "bench"), ring_steps=256)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e_start, e_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_up, e_run = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    g2.set_fields(pin_F.numpy(), None)
    for f, v in fault0.items():
        g2.set_fault(0, f, v)
    e_up.record(stream)
    lib().fdmap_gpu_init_edges(g2._g, host.t0)
    g2.run(1, args.steps, nt=nt_inf)
    if nf:
        g2.output_flush()
    e_run.record(stream)
    rc = lib().fdmap_gpu_get_fields(g2._g, C.cast(pin_out.data_ptr(), C.POINTER(C.c_double)), None)
    e_stop.record(stream)
    e_stop.synchronize()
    e_parts = {"upload_ms": e_start.elapsed_time(e_up), "steps_and_output_ms": e_up.elapsed_time(e_run),
               "download_ms": e_run.elapsed_time(e_stop)}
    if rc:
        raise RuntimeError(f"fdmap_gpu_get_fields failed ({rc})")
    e_ms = max(e_start.elapsed_time(e_stop), (time.perf_counter() - t0) * 1e3)
    e_ms = barrier_max(e_ms, world)
    e2e = world * nodes * args.steps / (e_ms * 1e-3)
    h2d = (F0.nbytes + sum(v.nbytes for v in fault0.values())) / args.steps
    d2h = (4 * nf * 4) + F0.nbytes / args.steps
    if nf:
        g2.output_close()
    g2.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(host, args)

    if rank == 0:
        ck = clocks.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": shared_config(info, host),
            "parallelism": f"replicas{world}",
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms": e_ms, **e_parts},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                         "frac": achieved / peaks["hbm_gbs"], "traffic": profiled_traffic(args.workload, kernel),
                         "kernel": kernel, "alg_bytes_per_launch": launch_bytes,
                         "alg_bytes_per_pass_launch": pass_bytes,
                         "alg_bytes_per_stage_launch": stage_bytes,
                         "mean_launch_ms": mean_ms,
                         "march_kernel": {"mean_launch_ms": stencil_ms if kn[0] else None, "achieved": march_gbs,
                                          "frac": march_gbs / peaks["hbm_gbs"] if march_gbs else None},
                         "closure_kernel_mean_ms": closure_ms, "interface_kernel_mean_ms": edge_ms,
                         "band_kernel_mean_ms": band_ms if kn[4] else None,
                         "peak_source": peaks["source"],
                         "step_level": {"achieved": step_gbs, "frac": step_gbs / peaks["hbm_gbs"],
                                        "bytes_per_step": sched_bytes,
                                        "stage_by_stage_bytes_per_node_update": bytes_per_node_update(
                                            host.mode, het, host.rk_order, host),
                                        "effective_stage_by_stage": unfused_gbs,
                                        "effective_frac": unfused_gbs / peaks["hbm_gbs"],
                                        "frac_without_metric_reads": survey_bytes / step_bytes * unfused_gbs
                                        / peaks["hbm_gbs"]}},
            "march_tile": tile_info,
            "two_stage_passes": pairs,
            "kernels_serialised": prof_kinds,
            "clocks": ck,
            "gpu_launches": launches,
            "newton_failures": newton_fail,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def interior_nodes(host) -> int:
    """Nodes handled by the interior kernel: all but the SBP closure strips."""
    nbst = {2: 1, 4: 4, 6: 6}
    fd = host.fd_method
    n = 0
    for b in range(host.nblocks):
        mgx, pgx, mgy, pgy = host.block_limits(b)
        nx, ny = pgx - mgx + 1, pgy - mgy + 1
        n += max(nx - 2 * nbst[fd], 0) * max(ny - 2 * nbst[fd], 0)
    return n


def lib_set_stream(g, stream) -> None:
    from fdmap_github_b200.native import check_gpu, lib

    check_gpu(lib().fdmap_gpu_set_stream(g._g, stream.cuda_stream), "fdmap_gpu_set_stream")


def cpu_baseline(host, args, seconds: float = 15.0) -> dict:
    """The oracle (CPU restatement of the reference's time step) on the host
    cores, timed on a bounded number of steps of the same workload."""
    from oracle.binding import OracleDomain, num_threads

    o = OracleDomain(host)
    o.run(1, 1, nt=1 << 30)  # warm-up step
    n, t0 = 0, time.perf_counter()
    while True:
        n += 1
        o.run(1 + n, 1 + n, nt=1 << 30)
        el = time.perf_counter() - t0
        if el > seconds or n >= 200:
            break
    nodes = host.nx * host.ny
    return {"value": nodes * n / el, "unit": UNIT, "cores": num_threads(), "kind": "port",
            "sample": f"{n} full LS-RK4 steps of the same {host.nx}x{host.ny}-node workload ({el:.1f} s)"}


def run_reference(args) -> None:
    """The CPU arm: the oracle (C++ restatement of the reference's time step;
    the Fortran/MPI reference cannot be built in this image) on the host
    cores, on the same workload, steps and warm-up as the GPU arm.  Its domain
    is set up by the host initialisation built on its own
    (oracle/_build/libhost_init.so), so no library of the GPU package loads."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    tmp = Path(tempfile.mkdtemp(prefix="fdmap_bench_ref_"))
    text, base, info = workload(args.workload, tmp)
    from oracle.binding import OracleDomain, init_domain_cpu, num_threads

    host = init_domain_cpu(text, base)
    o = OracleDomain(host)
    nodes = host.nx * host.ny
    nt_inf = 1 << 30
    o.run(1, args.warmup, nt=nt_inf)
    t0 = time.perf_counter()
    o.run(args.warmup + 1, args.warmup + args.steps, nt=nt_inf)
    el = time.perf_counter() - t0
    v = nodes * args.steps / el
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": shared_config(info, host),
            "parallelism": f"host threads ({num_threads()})",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": num_threads(), "kind": "port",
                             "sample": f"{args.steps} full LS-RK4 steps (after {args.warmup} warm-up steps) of the "
                                       f"same {host.nx}x{host.ny}-node workload ({el:.1f} s)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ensemble(args) -> None:
    """Batched ensemble (64 mode II rate-and-state instances of seeded grid
    sizes and von Karman prestress): runs/s of the ensemble against the same
    instances advanced one after another by the plain single-domain path.  A
    run is 1000 steps; both arms are timed on `--steps` steps after warm-up
    and scaled to the run length."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from fdmap_github_b200 import GpuEnsemble

    tmp = Path(tempfile.mkdtemp(prefix=f"fdmap_bench_ens_r{rank}_"))
    n = args.instances
    from fdmap_github_b200 import init_domains

    t_init = time.perf_counter()
    hosts = init_domains([problems.ensemble_instance(tmp, s) for s in range(n)], tmp)
    t_init = time.perf_counter() - t_init
    t_create = time.perf_counter()
    nodes = sum(h.nx * h.ny for h in hosts)
    dt = min(h.dt for h in hosts)
    run_steps = 1000
    ens = GpuEnsemble(hosts, device=local)
    ens.synchronize()
    t_create = time.perf_counter() - t_create
    shape, tune_ms = ens.tune(steps=5, dt=dt)
    tile = ens.tile
    ens.run(1, args.warmup, dt=dt, nt=1 << 30)
    ens.synchronize()
    barrier(world)
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        ens.run(args.warmup + 1, args.warmup + args.steps, dt=dt, nt=1 << 30)
        ens.synchronize()
        el = time.perf_counter() - t0
    launches = ens.launch_count()
    ens.close()
    el = barrier_max(el, world)
    # sequential arm: the same instances through the plain path, one at a time
    seq = 0.0
    for h in hosts:
        g = GpuDomain(h, device=local)
        g.tune(steps=2, dt=dt)  # each plain run with its own best tile, as the ensemble has its own
        g.run(1, args.warmup, dt=dt, nt=1 << 30)
        g.synchronize()
        t0 = time.perf_counter()
        g.run(args.warmup + 1, args.warmup + args.steps, dt=dt, nt=1 << 30)
        g.synchronize()
        seq += time.perf_counter() - t0
        g.close()
    # the same instances with their bodies built on the device (on-device init)
    t_init_dev = time.perf_counter()
    devs = init_domains([problems.ensemble_instance(tmp, s) for s in range(n)], tmp, body_on_device=True)
    t_init_dev = time.perf_counter() - t_init_dev
    t_create_dev = time.perf_counter()
    ens_dev = GpuEnsemble(devs, device=local)
    ens_dev.synchronize()
    t_create_dev = time.perf_counter() - t_create_dev
    same_dt = all(a.dt == b.dt for a, b in zip(devs, hosts))
    ens_dev.close()
    per_step = el / args.steps
    runs = world * n / (per_step * run_steps)
    if rank == 0:
        line = {"metric": "ensemble runs/s", "value": runs, "unit": "runs/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"{n} mode II rate-and-state instances (RFL), 2 blocks each of "
                                       "401x401 / 801x401 / 801x801 / 1601x801 (seeded), von Karman prestress",
                           "instances": n, "nodes": nodes, "run_steps": run_steps, "shape": list(shape),
                           "march_tile": tile,
                           "tuned_ms_per_step": tune_ms},
                "node_updates_per_s": world * nodes / per_step,
                "sequential_plain": {"runs_per_s": n / (seq / args.steps * run_steps),
                                     "ms_per_step": seq / args.steps * 1e3},
                "speedup_vs_sequential": seq / el, "host_init_s": t_init, "ensemble_create_s": t_create,
                "device_body_init": {"host_init_s": t_init_dev, "ensemble_create_s": t_create_dev,
                                     "same_dt_as_host_body": same_dt},
                "clocks": clocks.summary(), "gpu_launches": launches}
        print(json.dumps(line), flush=True)


def time_gradient(a, data, local, budget):
    """One warm-up forward-with-data + backward pair, then the timed pair, at
    the given stage-store budget (0: every segment recomputed from its
    checkpoint; -1: as many segments resident as device memory holds)."""
    a.set_store_budget(budget)
    a.forward(data=data)
    a.backward()
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        _, J = a.forward(data=data)
        t_af = time.perf_counter() - t0
        t0 = time.perf_counter()
        grads = a.backward()
        t_bwd = time.perf_counter() - t0
    grads = tuple(grads) + ((a.prestress_gradient(),) if a.fault_size else ())
    return {"forward_with_data_s": t_af, "backward_s": t_bwd, "misfit": J,
            "resident_segments": a.resident_segments,
            "store_gb": a.resident_segments * a.segment_bytes / 1e9, "clocks": clocks.summary()}, grads


def gradient_line(t_fwd, timed, recompute, same):
    """Keys shared by the adjoint lines: the resident-store timing is the
    headline, the recompute-everything timing is reported beside it."""
    return {"forward_s": t_fwd, "forward_with_data_s": timed["forward_with_data_s"],
            "backward_s": timed["backward_s"], "backward_over_forward": timed["backward_s"] / t_fwd,
            "forward_plus_backward_over_forward": (timed["forward_with_data_s"] + timed["backward_s"]) / t_fwd,
            "misfit": timed["misfit"], "resident_segments": timed["resident_segments"],
            "store_gb": round(timed["store_gb"], 2),
            "recompute_all": {"forward_with_data_s": recompute["forward_with_data_s"],
                              "backward_s": recompute["backward_s"],
                              "backward_over_forward": recompute["backward_s"] / t_fwd,
                              "forward_plus_backward_over_forward":
                                  (recompute["forward_with_data_s"] + recompute["backward_s"]) / t_fwd,
                              "clocks": recompute["clocks"]},
            "gradients_equal_bitwise": same, "clocks": timed["clocks"]}


def run_adjoint(args) -> None:
    """Forward/backward pair on the heterogeneous mode III block (801x801,
    2000 steps, 32 receivers on the top row, segments of 45 steps): the
    gradient's time (forward with data + backward) over one plain forward
    solve, with every segment's stage inputs resident in device memory (157
    GB) and, beside it, with every segment recomputed from its checkpoint;
    the two gradients compared bitwise, and 16 random-direction
    central-difference checks of the gradient (h = 1e-6 relative)."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from fdmap_github_b200 import GpuAdjoint

    tmp = Path(tempfile.mkdtemp(prefix=f"fdmap_bench_adj_r{rank}_"))
    host = init_domain(problems.heterogeneous_ricker(tmp), tmp)
    n = host.nx
    rec = [(int(i), host.ny) for i in np.linspace(2, n - 1, 32).round().astype(int)]
    rho, G = host.array("rho")[0].copy(), host.array("G")[0].copy()
    # plain forward solve of the same problem (the reference point of the ratio)
    g = GpuDomain(host, device=local)
    g.run(1, 3, nt=1 << 30)
    g.synchronize()
    t0 = time.perf_counter()
    g.run(1, host.nt - 1, nt=1 << 30)
    g.synchronize()
    t_fwd = time.perf_counter() - t0
    g.close()
    a = GpuAdjoint(host, rec, checkpoint_every=45, device=local)
    y, x = np.meshgrid(np.linspace(0, 1, host.ny), np.linspace(0, 1, host.nx), indexing="ij")
    bump = np.exp(-((x - 0.4) ** 2 + (y - 0.7) ** 2) / 0.02)
    a.set_material(rho * (1 + 0.05 * bump), G * (1 - 0.05 * bump))
    data, _ = a.forward()  # data: the perturbed model's seismograms
    a.set_material(rho, G)
    recompute, g_ref = time_gradient(a, data, local, 0)
    timed, (g_rho, g_G) = time_gradient(a, data, local, -1)
    same = all(np.array_equal(x, y) for x, y in zip(g_ref, (g_rho, g_G)))
    rng = np.random.default_rng(0)
    eps, errs = 1e-6, []
    for _ in range(16):
        d_rho = rng.uniform(-1, 1, rho.shape)
        d_G = rng.uniform(-1, 1, G.shape)
        pred = float(np.sum(g_rho * rho * d_rho) + np.sum(g_G * G * d_G))
        a.set_material(rho * (1 + eps * d_rho), G * (1 + eps * d_G))
        _, Jp = a.forward(data=data)
        a.set_material(rho * (1 - eps * d_rho), G * (1 - eps * d_G))
        _, Jm = a.forward(data=data)
        fd = (Jp - Jm) / (2 * eps)
        errs.append(abs(fd - pred) / abs(fd))
    a.close()
    if rank == 0:
        nodes = host.nx * host.ny
        g = gradient_line(t_fwd, timed, recompute, same)
        line = {"metric": "gradient/forward time", "value": g["forward_plus_backward_over_forward"],
                "unit": "ratio", "n_gpus": world, "steps": host.nt - 1, "warmup": 1,
                "ms_per_step": timed["backward_s"] / (host.nt - 1) * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "mode III heterogeneous 801x801 (dx 20 m), Ricker 5 Hz point force, "
                                       "32 top-row receivers, LS-RK4, segments of 45 steps, stage inputs "
                                       "resident in device memory",
                           "nodes": nodes, "steps": host.nt - 1},
                "forward_node_updates_per_s": nodes * (host.nt - 1) / t_fwd, **g,
                "fd_check": {"directions": 16, "h_rel": eps, "max_rel_err": max(errs),
                             "median_rel_err": float(np.median(errs))}}
        print(json.dumps(line), flush=True)


def run_adjoint_fault(args) -> None:
    """Forward/backward pair across a rate-and-state fault (aging law): two
    heterogeneous mode III blocks of 801x401 nodes (h = 25 m), 1000 steps, 32
    receivers two and three nodes off the fault, segments of 45 steps.  The
    gradient's time over one plain forward solve with the stage inputs
    resident and with every segment recomputed, and 4 random-direction
    central-difference checks in rho, G and the fault prestress together
    (h = 1e-6 relative)."""
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from fdmap_github_b200 import GpuAdjoint

    tmp = Path(tempfile.mkdtemp(prefix=f"fdmap_bench_adjf_r{rank}_"))
    host = init_domain(problems.heterogeneous_rs_fault(tmp, n=801, h=0.025, nt=1001, law="RAL"), tmp)
    m = host.ny // 2
    cols = np.linspace(3, host.nx - 2, 16).round().astype(int)
    rec = [(int(i), m - 2) for i in cols] + [(int(i), m + 4) for i in cols]
    rho, G = host.array("rho")[0].copy(), host.array("G")[0].copy()
    g = GpuDomain(host, device=local)
    g.run(1, 3, nt=1 << 30)
    g.synchronize()
    t0 = time.perf_counter()
    g.run(1, host.nt - 1, nt=1 << 30)
    g.synchronize()
    t_fwd = time.perf_counter() - t0
    g.close()
    a = GpuAdjoint(host, rec, checkpoint_every=45, device=local)
    nf = a.fault_size
    y, x = np.meshgrid(np.linspace(0, 1, host.ny), np.linspace(0, 1, host.nx), indexing="ij")
    bump = np.exp(-((x - 0.4) ** 2 + (y - 0.6) ** 2) / 0.02)
    s = np.linspace(-1, 1, nf)
    a.set_material(rho * (1 + 0.05 * bump), G * (1 - 0.05 * bump))
    a.set_prestress(2.0 * np.exp(-((s - 0.2) / 0.3) ** 2))
    data, _ = a.forward()
    a.set_material(rho, G)
    a.set_prestress(np.zeros(nf))
    recompute, g_ref = time_gradient(a, data, local, 0)
    timed, (g_rho, g_G, g_S0) = time_gradient(a, data, local, -1)
    same = all(np.array_equal(x, y) for x, y in zip(g_ref, (g_rho, g_G, g_S0)))
    rng = np.random.default_rng(0)
    eps, errs = 1e-6, []
    for _ in range(4):
        d_rho, d_G, d_S = rng.uniform(-1, 1, rho.shape), rng.uniform(-1, 1, G.shape), rng.uniform(-1, 1, nf)
        pred = float(np.sum(g_rho * rho * d_rho) + np.sum(g_G * G * d_G) + np.sum(g_S0 * 58.0 * d_S))
        Js = []
        for sg in (1, -1):
            a.set_material(rho * (1 + sg * eps * d_rho), G * (1 + sg * eps * d_G))
            a.set_prestress(sg * eps * 58.0 * d_S)
            Js.append(a.forward(data=data)[1])
        fd = (Js[0] - Js[1]) / (2 * eps)
        errs.append(abs(fd - pred) / abs(fd))
    a.close()
    if rank == 0:
        nodes = host.nx * host.ny
        g = gradient_line(t_fwd, timed, recompute, same)
        line = {"metric": "gradient/forward time", "value": g["forward_plus_backward_over_forward"],
                "unit": "ratio", "n_gpus": world, "steps": host.nt - 1, "warmup": 1,
                "ms_per_step": timed["backward_s"] / (host.nt - 1) * 1e3,
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "mode III rate-and-state fault (aging law) between two heterogeneous "
                                       "801x401 blocks (dx 25 m), 32 receivers beside the fault, LS-RK4, "
                                       "segments of 45 steps, stage inputs resident in device memory",
                           "nodes": nodes, "fault_nodes": nf, "steps": host.nt - 1},
                "forward_node_updates_per_s": nodes * (host.nt - 1) / t_fwd, **g,
                "fd_check": {"directions": 4, "h_rel": eps, "max_rel_err": max(errs),
                             "median_rel_err": float(np.median(errs))}}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--workload", default="rupture",
                    choices=["rupture", "pulse", "roughfault", "rupture_cdiss", "pml", "ensemble", "adjoint",
                             "adjoint_fault"])
    ap.add_argument("--instances", type=int, default=64, help="ensemble workload: number of instances")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "adjoint_fault":
        run_adjoint_fault(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
