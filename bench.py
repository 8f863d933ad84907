#!/usr/bin/env python3
"""Benchmark: the constant-coefficient ADI sweep on a 256^3 FP64 grid.

Workload (one "step"): one ADI run of 50 iterations, each iteration solving
the pentadiagonal systems along x, then y, then z of a 256^3 FP64 grid in
place, with the general kernels reading full coefficient arrays
(ds = dw = -r/12, dl = du = 16r/12, d = 1 + 30r/12, r = 0.5; initial field
U(-1,1) from a fixed seed).  Every solve goes through the library's C ABI
(libpentadsolver_b200.so), automatic kernel selection.

Metric: algorithmic HBM bandwidth, 7 arrays x 8 B = 56 B per grid point per
axis (5 coefficient arrays + RHS read, solution written), over the device
time of the step.  Inputs are 7 x 128 MiB per axis, larger than the 126 MB
L2, so no flush is needed between steps.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun every rank solves its own grid (independent replicas: the
path has no data exchange), timed with CUDA events between barriers; the
reported time is the max over ranks and `value` counts all ranks' bytes.
With --gpus N > 1 and no torchrun environment, the script launches N ranks
itself (torch.distributed.run on 127.0.0.1) with the same arguments.

--impl reference times the reference's own CPU solver (its AVX2 + OpenMP
src/cpu/singlenode/pentad_cpu.cpp, compiled from its sources into
oracle/_ref) on all host cores, each step the same 50-iteration ADI run.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
PKG = REPO / "pentadiagonal-solver_b200"
for p in (str(PKG), str(REPO)):
    if p not in sys.path:
        sys.path.insert(0, p)

N_DEFAULT = 256
ITERS = 50
EV_EVERY = 5  # iterations between timed launches (per-direction launch times)


def max_over_ranks(ms: float, world: int, device) -> float:
    """The slowest rank's time, on every rank (replicas finish when the last
    one does).  `device` holds the reduction tensor: the GPU under NCCL, the
    CPU under gloo."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_rank: float, ms: float, world: int) -> float:
    """GB/s of all ranks together: every replica moves `bytes_per_rank` in `ms`."""
    return world * bytes_per_rank / (ms * 1e-3) / 1e9


R_DIFF = 0.5
SEED = 2024
BYTES_PER_POINT_AXIS = 7 * 8
METRIC = "ADI sweep HBM GB/s (256^3 FP64, 50 x/y/z iterations per step)"


def peak_hbm():
    f = REPO / "MEASURED_PEAKS.json"
    try:
        v = float(json.loads(f.read_text())["hbm_gbs"])
        return v, "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_record():
    """Per-launch DRAM bytes of the solve kernels from the committed ncu
    summary (profiles/traffic.json), or None."""
    f = REPO / "profiles" / "traffic.json"
    try:
        return json.loads(f.read_text())
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        rows = []
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "max": float(parts[2]),
                             "power": float(parts[3]) if parts[3] not in ("[N/A]", "") else 0.0,
                             "hw": parts[5], "hwt": parts[6], "swt": parts[7], "pcap": parts[8]})
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [r for r in rows if r["power"] > 200.0] or rows
        reasons = set()
        for r in loaded:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in loaded),
                "sm_max_mhz": max(r["max"] for r in rows), "reasons": sorted(reasons),
                "samples": len(loaded)}


def adi_problem(n: int, device, dtype):
    import torch

    g = torch.Generator(device="cpu").manual_seed(SEED)
    shape = (n, n, n)
    field = (torch.rand(shape, generator=g, dtype=torch.float64) * 2.0 - 1.0).to(dtype)
    c = {
        "ds": -R_DIFF / 12.0, "dl": 16.0 * R_DIFF / 12.0, "d": 1.0 + 30.0 * R_DIFF / 12.0,
        "du": 16.0 * R_DIFF / 12.0, "dw": -R_DIFF / 12.0,
    }
    host = {k: torch.full(shape, v, dtype=dtype) for k, v in c.items()}
    host["x"] = field
    dev = {k: v.to(device) for k, v in host.items()}
    return host, dev


def spawn_ranks(n: int, argv: list[str]) -> int:
    """Run this script as `n` ranks under torch.distributed.run (one node,
    127.0.0.1, a free port) with the given arguments; returns the exit code
    (rank 0 prints the JSON line)."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve()), *argv]
    return subprocess.run(cmd).returncode


def reference_gpu_leg(d, names, n, iters=ITERS):
    """The reference's own GPU solver (src/cuda/singlenode/pentad_cuda.cu built
    for sm_100a, stock dispatch) on the same grid and coefficients: `iters`
    ADI iterations timed with CUDA events on the legacy default stream it
    launches on.  Outside every timed region of this bench."""
    import ctypes

    import torch

    from oracle import oracle

    if not oracle.ref_available("cuda"):
        return {"unavailable": "oracle/_ref/libpentad_cuda_ref.so not built"}
    solve, ran = oracle.ref_cuda_solver()
    x = d["x"].clone()
    buf = torch.empty(9 * n ** 3 * 8, dtype=torch.uint8, device=x.device)  # its x sizing
    cdims = (ctypes.c_int * 3)(n, n, n)
    ptrs = [ctypes.c_void_p(d[k].data_ptr()) for k in names] + [ctypes.c_void_p(x.data_ptr())]
    bp = ctypes.c_void_p(buf.data_ptr())
    legacy = torch.cuda.default_stream(x.device)
    torch.cuda.synchronize()
    with torch.cuda.stream(legacy):
        for axis in range(3):   # warm-up: module load, first launches
            solve(None, *ptrs, cdims, 3, axis, bp)
        torch.cuda.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(iters)]
        for it in range(iters):
            for axis in range(3):
                ev[it][axis].record(legacy)
                solve(None, *ptrs, cdims, 3, axis, bp)
            ev[it][3].record(legacy)
        torch.cuda.synchronize()
    per_dir = [statistics.mean(ev[it][a].elapsed_time(ev[it][a + 1]) for it in range(iters))
               for a in range(3)]
    ms_it = ev[0][0].elapsed_time(ev[-1][3]) / iters
    del buf
    return {"value": round(BYTES_PER_POINT_AXIS * n ** 3 * 3 / (ms_it * 1e-3) / 1e9, 1),
            "unit": "GB/s", "ms_per_iteration": round(ms_it, 4),
            "per_direction_ms": [round(v, 4) for v in per_dir],
            "kernels": [ran(a) for a in range(3)], "iterations": iters,
            "what": "src/cuda/singlenode/pentad_cuda.cu (sm_100a, stock dispatch), same "
                    "grid, coefficients and field; CUDA events on its launch stream"}


def run_ours(args):
    import torch
    import torch.distributed as dist

    import pentadsolver as ps

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.n
    dims = [n, n, n]
    host, d = adi_problem(n, dev, torch.float64)
    names = ("ds", "dl", "d", "du", "dw")
    buf = ps.alloc_buffer(dims, 0, torch.float64, dev)
    stream = torch.cuda.Stream(device=dev)
    handle = ps.Handle()

    def solve(axis, x):
        ps.gpsv_batch(*(d[k] for k in names), x, axis, buffer=buf, stream=stream,
                      handle=handle)

    def step(x, dir_events=None):
        for it in range(ITERS):
            timed_it = dir_events is not None and it % EV_EVERY == 0
            for axis in range(3):
                if timed_it:
                    dir_events[it // EV_EVERY][axis][0].record(stream)
                solve(axis, x)
                if timed_it:
                    dir_events[it // EV_EVERY][axis][1].record(stream)

    x = d["x"]
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(x)
    stream.synchronize()
    ran = [handle.kernel_that_ran(a) for a in range(3)]
    variants = [handle.variant_that_ran(a) for a in range(3)]

    # ---- timed region: K steps, device time ---------------------------------
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    # an event pair around every launch of every EV_EVERY-th iteration of the
    # timed region (average launch duration per direction, for the roofline;
    # sampled so that the records add little to the step time)
    dir_ev = [[[[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(3)]
               for _ in range(ITERS // EV_EVERY)] for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for k in range(args.steps):
            step(x, dir_ev[k])
        ev1.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    ms_total = ev0.elapsed_time(ev1)
    ms_total = max_over_ranks(ms_total, world, dev)
    if world > 1:
        dist.barrier()
    ms_step = ms_total / args.steps
    per_dir_ms = [statistics.mean(dir_ev[k][j][a][0].elapsed_time(dir_ev[k][j][a][1])
                                  for k in range(args.steps) for j in range(ITERS // EV_EVERY))
                  for a in range(3)]
    alg_bytes_step = BYTES_PER_POINT_AXIS * n ** 3 * 3 * ITERS
    value = whole_job_gbs(alg_bytes_step, ms_step, world)

    # ---- the same steps, each one CUDA graph of its 150 solves ----------------
    from adi import AdiGraph

    adi_graph = AdiGraph(*(d[k] for k in names), d["x"], iterations=ITERS, buffer=buf,
                         handle=handle)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            adi_graph.replay()
    torch.cuda.synchronize()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        g0.record(stream)
        for _ in range(args.steps):
            adi_graph.replay()
        g1.record(stream)
    torch.cuda.synchronize()
    graph_ms = g0.elapsed_time(g1) / args.steps
    graph_ms = max_over_ranks(graph_ms, world, dev)
    adi_graph.close()
    del adi_graph

    # ---- end to end through the public API with host buffers ----------------
    # Every step is a fresh problem: its six arrays come from pinned host
    # memory and its result goes back.  Steps are pipelined as a serving loop
    # would run them: two device sets of the arrays; the host->device copies
    # of step k+1 (one copy stream) and the read-back of step k-1 (another)
    # overlap the solves of step k.  The timed region spans the first copy in
    # to the last copy out, over the same K steps as the device-timed value
    # (the first copy in and the last copy out overlap nothing).
    pinned = {k: v.pin_memory() for k, v in host.items()}
    out = torch.empty_like(pinned["x"]).pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in pinned.values())
    d2h = out.numel() * out.element_size()
    e2e_steps = max(3, args.steps)
    sets = [d, {k: torch.empty_like(v) for k, v in d.items()}]
    s_in = torch.cuda.Stream(device=dev)
    s_out = torch.cuda.Stream(device=dev)
    loaded = [torch.cuda.Event() for _ in range(2)]
    solved = [torch.cuda.Event() for _ in range(2)]
    freed = [torch.cuda.Event() for _ in range(2)]

    def solve_set(axis, S):
        ps.gpsv_batch(*(S[k] for k in names), S["x"], axis, buffer=buf, stream=stream,
                      handle=handle)

    def load(i):
        S = sets[i % 2]
        with torch.cuda.stream(s_in):
            if i >= 2:
                s_in.wait_event(freed[i % 2])  # step i-2's result has left this set
            for k in ("ds", "dl", "d", "du", "dw", "x"):
                S[k].copy_(pinned[k], non_blocking=True)
            loaded[i % 2].record(s_in)

    def e2e_run(steps):
        load(0)
        for i in range(steps):
            S = sets[i % 2]
            stream.wait_event(loaded[i % 2])
            for it in range(ITERS):
                for axis in range(3):
                    solve_set(axis, S)
            solved[i % 2].record(stream)
            if i + 1 < steps:
                load(i + 1)
            with torch.cuda.stream(s_out):
                s_out.wait_event(solved[i % 2])
                out.copy_(S["x"], non_blocking=True)
                freed[i % 2].record(s_out)
        stream.wait_stream(s_out)

    e2e_run(2)  # warm-up of the pipeline
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    e2e_run(e2e_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    e2e_value = whole_job_gbs(alg_bytes_step, e2e_ms, world)

    # ---- one solve per step, end to end: what a single call on host buffers
    # costs (the copies dominate: 48 B/pt in, 8 B/pt out over PCIe, against
    # 56 B/pt of HBM traffic for the solve itself); x direction, serialised
    def single_call_run(reps):
        S = sets[0]
        for _ in range(reps):
            with torch.cuda.stream(stream):
                for k in ("ds", "dl", "d", "du", "dw", "x"):
                    S[k].copy_(pinned[k], non_blocking=True)
                solve_set(0, S)
                out.copy_(S["x"], non_blocking=True)

    single_call_run(2)
    torch.cuda.synchronize()
    c0 = torch.cuda.Event(enable_timing=True)
    c1 = torch.cuda.Event(enable_timing=True)
    single_reps = max(3, min(args.steps, 10))
    c0.record(stream)
    single_call_run(single_reps)
    c1.record(stream)
    torch.cuda.synchronize()
    single_ms = c0.elapsed_time(c1) / single_reps
    single_ms = max_over_ranks(single_ms, world, dev)
    single_value = whole_job_gbs(BYTES_PER_POINT_AXIS * n ** 3, single_ms, world)

    # ---- roofline of the dominant kernel -------------------------------------
    # The dominant kernel is the instantiation with the largest share of the
    # timed solves (directions that ran the same variant are one kernel); its
    # average launch duration is the mean over those directions.  The slowest
    # direction is reported beside it.
    groups: dict[str, list[int]] = {}
    for a in range(3):
        groups.setdefault(variants[a], []).append(a)
    dom_dirs = max(groups.values(), key=lambda dirs: sum(per_dir_ms[a] for a in dirs))
    dom_ms = sum(per_dir_ms[a] for a in dom_dirs) / len(dom_dirs)
    share = sum(per_dir_ms[a] for a in dom_dirs) / sum(per_dir_ms)
    alg_launch = BYTES_PER_POINT_AXIS * n ** 3
    achieved = alg_launch / (dom_ms * 1e-3) / 1e9
    slow = max(range(3), key=lambda a: per_dir_ms[a])
    slow_achieved = alg_launch / (per_dir_ms[slow] * 1e-3) / 1e9
    peak, peak_src = peak_hbm()
    tr = traffic_record()

    def traffic_of(dirs):
        if tr is None:
            return None
        vals = []
        for a in dirs:
            rec = tr.get(f"dir{a}")
            if rec is None or rec.get("n") != n or rec.get("variant") != variants[a]:
                return None
            vals.append(rec.get("bytes_per_launch"))
        return int(sum(vals) / len(vals))

    traffic = traffic_of(dom_dirs)

    result = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (config 1 coefficients, seeded U(-1,1) field)",
        "config": {
            "workload": "adi_256cube_fp64_general_50iter",
            "grid": dims,
            "iters_per_step": ITERS,
            "kernel_family": ran,
            "kernel_variant": variants,
            "per_direction_ms": [round(v, 4) for v in per_dir_ms],
            "ms_per_iteration": round(ms_step / ITERS, 4),
            "systems_per_s": round(world * 3 * ITERS * n * n / (ms_step * 1e-3), 1),
            "l2": "no flush: 7 x 128 MiB per axis exceeds the 126 MB L2",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        },
        "clocks": clk.summary(),
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_ms, 3),
                "steps": e2e_steps,
                "schedule": "pipelined: copies in of step k+1 and out of step k-1 overlap "
                            "the solves of step k (two device sets, two copy streams)"},
        "e2e_single_call": {"value": round(single_value, 2), "unit": "GB/s",
                            "ms_per_call": round(single_ms, 3), "h2d_bytes_per_call": h2d,
                            "d2h_bytes_per_call": d2h, "calls": single_reps,
                            "note": "one x solve per call: six arrays in from pinned host "
                                    "memory, solve, result out, serialised on one stream"},
        "graph": {"value": round(whole_job_gbs(alg_bytes_step, graph_ms, world), 2),
                  "unit": "GB/s", "ms_per_step": round(graph_ms, 4),
                  "note": "each step's 150 solves replayed as one CUDA graph (adi.AdiGraph)"},
        "gpu_launches": args.steps * ITERS * 3,
        "roofline": {
            "bound": "hbm",
            "kernel": f"{variants[dom_dirs[0]]} (dir {', '.join(str(a) for a in dom_dirs)})",
            "share_of_solve_time": round(share, 3),
            "achieved": round(achieved, 1),
            "peak": peak,
            "peak_source": peak_src,
            "unit": "GB/s",
            "frac": round(achieved / peak, 4),
            "traffic": traffic,
            "algorithmic_bytes_per_launch": alg_launch,
            "slowest_direction": {"dir": slow, "kernel": variants[slow],
                                  "achieved": round(slow_achieved, 1),
                                  "frac": round(slow_achieved / peak, 4),
                                  "traffic": traffic_of([slow])},
        },
    }
    # ---- the reference's own GPU path on the same problem (not timed above) --
    if world == 1 and not args.no_reference_gpu:
        result["reference_gpu"] = reference_gpu_leg(d, names, n)
        if "ms_per_iteration" in result["reference_gpu"]:
            result["reference_gpu"]["our_speedup"] = round(
                result["reference_gpu"]["ms_per_iteration"] / (ms_step / ITERS), 2)

    # ---- the same ADI run with shared factorisation (constant coefficients) --
    # Algorithmic bytes: RHS read + solution written, 2 x 8 B per point per
    # axis (the 5n-entry table is negligible).  Same field, same 50 x 3 solves.
    sf_handle = ps.Handle()
    for a in range(3):
        sf_handle.set_algo(a, "shared-fact")
    x.copy_(host["x"])

    def sf_step():
        for it in range(ITERS):
            for axis in range(3):
                ps.gpsv_batch(*(d[k] for k in names), x, axis, buffer=buf, stream=stream,
                              handle=sf_handle)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            sf_step()
    stream.synchronize()
    if world > 1:
        dist.barrier()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    sf_steps = max(1, min(args.steps, 10))
    with torch.cuda.stream(stream):
        s0.record(stream)
        for _ in range(sf_steps):
            sf_step()
        s1.record(stream)
    stream.synchronize()
    sf_ms = s0.elapsed_time(s1) / sf_steps
    sf_ms = max_over_ranks(sf_ms, world, dev)
    sf_bytes = 2 * 8 * n ** 3 * 3 * ITERS
    sf_gbs = whole_job_gbs(sf_bytes, sf_ms, world)
    result["shared_fact"] = {
        "value": round(sf_gbs, 2), "unit": "GB/s", "ms_per_step": round(sf_ms, 4),
        "bytes_per_point_axis": 16, "frac_of_peak": round(sf_gbs / world / peak, 4),
        "kernel_variant": [sf_handle.variant_that_ran(a) for a in range(3)],
        "systems_per_s": round(world * 3 * ITERS * n * n / (sf_ms * 1e-3), 1),
    }
    sf_handle.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(n, budget_s=args.cpu_seconds)
    handle.close()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(result))


def _cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_problem(n):
    import numpy as np

    rng = np.random.default_rng(SEED)
    shape = (n, n, n)
    co = {
        "ds": np.full(shape, -R_DIFF / 12.0), "dl": np.full(shape, 16.0 * R_DIFF / 12.0),
        "d": np.full(shape, 1.0 + 30.0 * R_DIFF / 12.0), "du": np.full(shape, 16.0 * R_DIFF / 12.0),
        "dw": np.full(shape, -R_DIFF / 12.0), "x": rng.uniform(-1.0, 1.0, shape),
    }
    return co


def cpu_solver():
    """The reference's own CPU solver (compiled from its tree into oracle/_ref)
    or, when that build is absent, the oracle port."""
    from oracle import oracle

    if oracle.ref_available("simd"):
        return (lambda co, axis: oracle.ref_solve(co["ds"], co["dl"], co["d"], co["du"],
                                                  co["dw"], co["x"], axis, which="simd"),
                "reference", "src/cpu/singlenode/pentad_cpu.cpp (OpenMP+AVX2)")
    return (lambda co, axis: oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"],
                                          co["x"], axis),
            "port", "oracle/penta_oracle.c")


def _cpu_sample(co, fn, threads, budget_s, max_iters=1000):
    """Whole ADI iterations of the CPU solver with `threads` OpenMP threads for
    about budget_s seconds: (iterations, seconds)."""
    from oracle import oracle

    oracle.set_threads(threads)
    for axis in range(3):  # warm-up (page faults, thread pool)
        fn(co, axis)
    t0 = time.perf_counter()
    iters = 0
    while iters < max_iters and (time.perf_counter() - t0) < budget_s:
        for axis in range(3):
            fn(co, axis)
        iters += 1
    return iters, time.perf_counter() - t0


def cpu_baseline(n, budget_s=12.0, single_s=4.0):
    """The reference's CPU solver on the host cores for about budget_s seconds
    of whole ADI iterations (the bounded sample the line reports), and again
    with one thread for about single_s seconds."""
    from oracle import oracle

    threads = _cpu_threads()
    co = cpu_problem(n)
    fn, kind, what = cpu_solver()
    iters, dt = _cpu_sample(co, fn, threads, budget_s)
    gbs = BYTES_PER_POINT_AXIS * n ** 3 * 3 * iters / dt / 1e9
    it1, dt1 = _cpu_sample(co, fn, 1, single_s)
    gbs1 = BYTES_PER_POINT_AXIS * n ** 3 * 3 * it1 / dt1 / 1e9
    oracle.set_threads(threads)
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": threads, "kind": kind,
            "cpu_model": oracle.cpu_model(), "nproc": os.cpu_count(),
            "sample": f"{iters} ADI iterations (x,y,z) of the {n}^3 FP64 grid, {what}, "
                      f"{threads} threads, {dt:.1f} s",
            "single_thread": {"value": round(gbs1, 3), "unit": "GB/s", "cores": 1,
                              "ms_per_iteration": round(dt1 * 1e3 / max(it1, 1), 1),
                              "sample": f"{it1} ADI iterations, 1 thread, {dt1:.1f} s"}}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle

    threads = _cpu_threads()
    oracle.set_threads(threads)
    n = args.n
    co = cpu_problem(n)
    fn, kind, what = cpu_solver()

    def step():  # one ADI run: 50 iterations of x, y, z, as the GPU arm's step
        for _ in range(ITERS):
            for axis in range(3):
                fn(co, axis)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    ms_step = dt * 1e3 / args.steps
    value = BYTES_PER_POINT_AXIS * n ** 3 * 3 * ITERS / (ms_step * 1e-3) / 1e9
    world = int(os.environ.get("WORLD_SIZE", "1"))
    print(json.dumps({
        "impl": "reference",
        "metric": METRIC,
        "value": round(value, 3),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms_step, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (config 1 coefficients, seeded U(-1,1) field)",
        "config": {"workload": "adi_256cube_fp64_general_50iter", "grid": [n, n, n],
                   "iters_per_step": ITERS,
                   "step": "one ADI run of 50 iterations (x,y,z), host cores",
                   "ms_per_iteration": round(ms_step / ITERS, 3),
                   "parallelism": "host cores"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GB/s", "cores": threads,
                         "kind": kind, "cpu_model": oracle.cpu_model(),
                         "nproc": os.cpu_count(),
                         "sample": f"{args.steps} ADI runs of {ITERS} iterations, {what}"},
        "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--grid-edge", dest="n", type=int, default=N_DEFAULT,
                    help="edge of the cubic grid (default 256)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus, sys.argv[1:]))
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
