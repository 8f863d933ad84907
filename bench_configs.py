#!/usr/bin/env python3
"""Measurements of the solver's other workloads, one JSON line each.

  config0  64^3 FP64, random dominant coefficients, x then y then z: time per
           axis and forward error against the CPU oracle (parity workload).
  config2  512^3 random dominant coefficients: plain FP64 against FP32 sweeps
           with 1..3 FP64 refinement steps; time, GB/s (56 B per point and
           axis for both: the same useful work) and forward error of every
           result against the FP64 CPU oracle, on every axis.
  config3  96 grids, N_x, N_y, N_z ~ U[32, 384] (seeded), random dominant
           coefficients, x, y and z each one plan (one persistent launch),
           the three captured in one CUDA graph; FP64 and FP32 + 1 refinement
           step (all 96 grids; casting the coefficients to FP32 in every execute,
           and keeping the copies of an earlier execute); against per-grid
           single calls.  Forward errors
           of both forms against the CPU oracle, grid by grid.
  refine1  one-step refined solves of config 2's 512^3 grid, 3 timed calls per axis
           (FP32 coefficient copies cached): the launch-list command.
  3split   config 3's FP64 plans per axis and bucket of line length along it (32-64
           ... 321-384, and all): where the time goes.
  config4  serving: a Poisson stream (2000 requests/s) of grids with per-axis
           N ~ logU[16, 512] from a device-resident pool, solvedim U{0,1,2},
           70% at tolerance 1e-10 and 30% at 1e-13, 150 GB budget; p50/p99
           latency and solves/s for the mixed and FP64 policies and for
           sequential plain FP64 calls, at that rate and at saturation; the
           mixed policy first measures, per solve direction, whether the
           refined form beats plain FP64 and uses it only where it does.  Each
           policy runs twice: the Python loop (serving.serve) and the library's
           native serving handle (serving.serve_native, pentadsolver_server_*).

  odd      odd-size grids: each axis of 255^3 against 256^3, FP64 and FP32, timed as
           single solves (CUDA events, 7 x 930 MB per axis: above L2, no flush),
           with the misaligned rows / runs loaded by 16-byte cp.async chunks
           (default), element copies (PENTA_TMEM_LOADS=element) and group-view
           TMA boxes (=group), aligned 256^3 also by bulk copies (=bulk), and the
           16 smallest of config 3's grids as FP64 plans; GB/s of 7 sizeof(F) B
           per point.

  mesh     the reference's random benchmark grid, 256^3 FP64 (the largest of
           benchmarks/cuda/my_bm.cu), built on the device by
           pentadsolver_D_mesh_random for several host thread counts, against
           the reference's own path: Mesh<double>(2, dims) on the host cores
           (include/util/mesh.hpp:85-124, compiled from the reference tree
           into oracle/_ref) with the same thread count, then the upload of
           its six arrays from pageable memory (device_mesh.hpp:52-65).  The
           device grid is compared with the reference's bit for bit.

  refapp   the reference's own ADI benchmark, apps/adi_cuda.cu unchanged, 256^3,
           50 timed iterations after its 1.5 s warm-up, built twice by
           oracle/Makefile: on the reference's GPU solver (app_cuda_ref) and on
           this library (app_cuda_b200); FP64 and FP32 with the default
           selectors, and FP64 with shared factorisation.  Its constant
           coefficients (1, 1, 5, 1, 1; RHS 1) are the app's own.  GB/s =
           algorithmic bytes of the three solves per iteration over the app's
           CUDA-event iteration time.

All inputs are synthetic (seeded); times are CUDA-event device times except
the serving loop and the reference's host mesh build (wall clock).  Every line
carries the SM clocks and throttle reasons sampled (nvidia-smi) while it ran.  Like
bench.py, this script uses oracle/ only as the checker (forward errors) and
for the reference's own CPU code timed as the baseline; the solves and grids
it measures are the library's.

  python bench_configs.py [--configs 0,2,refine1,3,3split,4,odd,mesh,refapp]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
HERE = REPO / "pentadiagonal-solver_b200"
for p in (str(HERE), str(REPO), str(REPO / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

NAMES = ("ds", "dl", "d", "du", "dw", "x")


def peak():
    try:
        return float(json.loads((REPO / "MEASURED_PEAKS.json").read_text())["hbm_gbs"])
    except Exception:
        return 6650.0


def dev_problem(dims, seed, dtype=None):
    """Random dominant problem (config-0 distribution) generated on the GPU."""
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    shape = tuple(reversed(list(dims)))

    def u(lo, hi):
        return torch.rand(shape, generator=g, device="cuda", dtype=torch.float64) * (hi - lo) + lo

    ds, dl, du, dw = u(-1, 1), u(-1, 1), u(-1, 1), u(-1, 1)
    d = ds.abs() + dl.abs() + du.abs() + dw.abs() + u(1, 2)
    out = {"ds": ds, "dl": dl, "d": d, "du": du, "dw": dw, "x": u(-1, 1)}
    if dtype is not None:
        out = {k: v.to(dtype) for k, v in out.items()}
    return out


def timed(fn, reps=3, warmup=1):
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def fwd_err(a, b) -> float:
    import torch

    a = a.double()
    b = b.double()
    return float((a - b).abs().max() / b.abs().max())


def oracle_errors(grids, rhs, results, axes):
    """Largest forward error of `results` against the CPU oracle solving each
    grid's right-hand side along `axes` in turn (grid by grid, so the host
    holds one grid at a time)."""
    import os

    from oracle import oracle

    oracle.set_threads(os.cpu_count() or 1)
    worst = 0.0
    for g, r, got in zip(grids, rhs, results):
        host = {k: g[k].cpu().numpy() for k in ("ds", "dl", "d", "du", "dw")}
        x = r.cpu().numpy()
        for axis in axes:
            oracle.solve(host["ds"], host["dl"], host["d"], host["du"], host["dw"], x, axis)
        xg = got.cpu().numpy()
        worst = max(worst, float(np.abs(xg - x).max() / np.abs(x).max()))
    return worst


def config0():
    import torch

    import fixtures
    import pentadsolver as ps
    from oracle import oracle

    dims = (64, 64, 64)
    co = fixtures.random_dominant(dims, 20240601, np.float64)
    dv = {k: torch.from_numpy(co[k]).cuda() for k in NAMES}
    ref = co["x"].copy()
    per_axis, errs = [], []
    with ps.Handle() as h:
        for axis in range(3):
            x0 = dv["x"].clone()
            ms = timed(lambda: (dv["x"].copy_(x0), ps.gpsv_batch(*(dv[k] for k in NAMES), axis,
                                                                  handle=h)),
                       reps=100, warmup=10)
            dv["x"].copy_(x0)
            ps.gpsv_batch(*(dv[k] for k in NAMES), axis, handle=h)
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
            errs.append(float(np.abs(dv["x"].cpu().numpy() - ref).max() / np.abs(ref).max()))
            per_axis.append(round(ms * 1e3, 2))
    return {"config": "config0_64cube_fp64_xyz", "us_per_axis_incl_copy": per_axis,
            "fwd_err_vs_oracle": errs, "tolerance": 1e-12,
            "note": "L2-resident parity workload (14 MiB per axis)"}


def config2(n=512):
    import torch

    import pentadsolver as ps
    from oracle import oracle

    dims = (n, n, n)
    p = dev_problem(dims, 2)
    b = p["x"].clone()
    pts = n ** 3
    out = {"config": f"config2_{n}cube_precision", "points": pts, "axes": []}
    with ps.Handle() as h:
        for axis in range(3):
            buf = ps.alloc_buffer(list(dims), axis, torch.float64)
            x64 = b.clone()

            def plain():
                x64.copy_(b)
                ps.gpsv_batch(p["ds"], p["dl"], p["d"], p["du"], p["dw"], x64, axis, buffer=buf,
                              handle=h)

            ms64 = timed(plain)
            copy_ms = timed(lambda: x64.copy_(b))
            plain()
            torch.cuda.synchronize()
            # the CPU FP64 oracle on this axis (the reference for every error)
            host = {k: p[k].cpu().numpy() for k in ("ds", "dl", "d", "du", "dw")}
            xr = b.cpu().numpy()
            oracle.set_threads(__import__("os").cpu_count() or 1)
            oracle.solve(host["ds"], host["dl"], host["d"], host["du"], host["dw"], xr, axis)
            ref = torch.from_numpy(xr).cuda()
            err_kind = "cpu_oracle"
            del host, xr
            row = {"axis": axis, "fp64": {"ms": round(ms64 - copy_ms, 4),
                                          "variant": h.variant_that_ran(0 if axis == 0 else (2 if axis == 2 else 1)),
                                          "fwd_err": fwd_err(x64, ref)}}
            del buf
            rbuf = ps.alloc_refine_buffer(list(dims), axis)
            xm = b.clone()
            for steps in (0, 1, 2, 3):
                def mixed(steps=steps, reuse=True):
                    xm.copy_(b)
                    ps.gpsv_batch_refine(p["ds"], p["dl"], p["d"], p["du"], p["dw"], xm, axis,
                                         steps=steps, buffer=rbuf, reuse_fp32_coefficients=reuse,
                                         handle=h)

                mixed(reuse=False)   # cast the coefficients once
                ms = timed(mixed) - copy_ms
                mixed()
                torch.cuda.synchronize()
                dmax, xmax = ps.refine_estimate(rbuf)
                row[f"fp32_ir{steps}"] = {"ms": round(ms, 4), "fwd_err": fwd_err(xm, ref),
                                          "estimate": dmax / xmax if xmax else None}
            # the cast itself (when coefficients change per solve)
            row["fp32_cast_ms"] = round(timed(lambda: mixed(1, False)) - timed(lambda: mixed(1, True)), 4)
            del rbuf
            row["fp64"]["GBps"] = round(56 * pts / (row["fp64"]["ms"] * 1e-3) / 1e9, 1)
            for s in (1, 2, 3):
                k = f"fp32_ir{s}"
                row[k]["GBps_equiv"] = round(56 * pts / (row[k]["ms"] * 1e-3) / 1e9, 1)
                row[k]["speed_vs_fp64"] = round(row["fp64"]["ms"] / row[k]["ms"], 3)
            row["fwd_err_reference"] = err_kind
            out["axes"].append(row)
            torch.cuda.empty_cache()
    out["peak_GBps"] = peak()
    out["target_fwd_err"] = 1e-10
    return out


def config3(n_grids=96, lo=32, hi=384, seed=33):
    import torch

    import pentadsolver as ps

    rng = np.random.default_rng(seed)
    dims_list = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(n_grids)]
    pts = sum(math.prod(d) for d in dims_list)
    grids = [dev_problem(d, 1000 + i) for i, d in enumerate(dims_list)]
    rhs = [g["x"].clone() for g in grids]
    out = {"config": "config3_batched_uneven", "grids": n_grids, "points": pts,
           "N_range": [lo, hi], "seed": seed}

    def restore():
        for g, r in zip(grids, rhs):
            g["x"].copy_(r)

    restore_ms = timed(restore)
    # the library's autotuner picks each plan's CTA count (recorded in its
    # tuning table, which plan creation with ctas = 0 then consults)
    import autotune

    tuner = autotune.Autotuner(reps=3)
    out["tuned_ctas_fp64"] = [tuner.tune_plan(grids, axis)["best"]["ctas"] for axis in range(3)]
    torch.cuda.empty_cache()
    # FP64 plans, captured together; the three share one scratch region
    shared = ps.aligned_bytes(max(ps.plan_sizes(grids, a)[1] for a in range(3)))
    plans = [ps.Plan(grids, axis, scratch=shared) for axis in range(3)]
    out["fp64_plans"] = [pl.describe() for pl in plans]
    s = torch.cuda.Stream()
    restore()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        for pl in plans:
            pl.execute(s)
    ms = timed(lambda: (restore(), graph.replay())) - restore_ms
    restore()
    graph.replay()
    torch.cuda.synchronize()
    ref = [g["x"].clone() for g in grids]
    out["fp64_fwd_err_max_vs_oracle"] = oracle_errors(grids, rhs, ref, axes=(0, 1, 2))
    out["fp64_graph_ms_xyz"] = round(ms, 3)
    out["fp64_GBps"] = round(3 * 56 * pts / (ms * 1e-3) / 1e9, 1)
    out["fp64_systems_per_s"] = round(sum(3 * math.prod(d) / max(d) for d in dims_list) / (ms * 1e-3))
    del graph
    for pl in plans:
        pl.close()
    del plans, shared
    torch.cuda.empty_cache()
    # sequential single calls (one launch per grid and axis, one stream, one
    # buffer sized for the largest grid)
    with ps.Handle() as h:
        buf = ps.aligned_bytes(max(ps.buffer_size(list(d), 0, 8) for d in dims_list))

        def singles():
            for g in grids:
                for axis in range(3):
                    ps.gpsv_batch(g["ds"], g["dl"], g["d"], g["du"], g["dw"], g["x"], axis,
                                  buffer=buf, handle=h)

        ms_single = timed(lambda: (restore(), singles())) - restore_ms
    del buf
    torch.cuda.empty_cache()
    out["single_calls_ms_xyz"] = round(ms_single, 3)
    out["batched_speedup"] = round(ms_single / ms, 3)
    # FP32 sweeps + 1 refinement step: one refinement plan per axis (its FP32
    # copies of the coefficients live in its own buffer), each axis captured
    # in a graph and timed, over all grids (x, y, z in turn, as FP64 above)
    ir_grids = n_grids
    sub, sub_rhs, sub_ref = grids[:ir_grids], rhs[:ir_grids], ref[:ir_grids]
    pts_ir = sum(math.prod(d) for d in dims_list[:ir_grids])
    out["ir1_grids"] = ir_grids
    try:
        for g, r in zip(sub, sub_rhs):
            g["x"].copy_(r)
        ms_axes, ms_reuse = [], []
        out["tuned_ctas_ir1"] = []
        for axis in range(3):
            out["tuned_ctas_ir1"].append(tuner.tune_plan(sub, axis, refine_steps=1)["best"]["ctas"])
            torch.cuda.empty_cache()
            rp = ps.Plan(sub, axis, refine_steps=1)
            saved = [g["x"].clone() for g in sub]

            def put_back():
                for g, sv in zip(sub, saved):
                    g["x"].copy_(sv)

            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=s):
                rp.execute(s)
            ms_axes.append(timed(lambda: (put_back(), graph.replay())) - timed(put_back))
            # the same with the FP32 copies kept from the executes above (fixed
            # coefficients, as in an ADI loop)
            graph_r = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph_r, stream=s):
                rp.execute(s, reuse_fp32=True)
            ms_reuse.append(timed(lambda: (put_back(), graph_r.replay())) - timed(put_back))
            del graph_r
            put_back()
            graph.replay()           # leave this axis solved, then the next axis
            torch.cuda.synchronize()
            del graph, saved
            rp.close()
            del rp
            torch.cuda.empty_cache()
        ms_r = sum(ms_axes)
        out["ir1_ms_xyz"] = round(ms_r, 3)
        out["ir1_ms_per_axis"] = [round(v, 3) for v in ms_axes]
        out["ir1_cached_fp32_ms_xyz"] = round(sum(ms_reuse), 3)
        out["ir1_cached_fp32_ms_per_axis"] = [round(v, 3) for v in ms_reuse]
        out["ir1_GBps_equiv"] = round(3 * 56 * pts_ir / (ms_r * 1e-3) / 1e9, 1)
        out["ir1_fwd_err_max_vs_oracle"] = oracle_errors(sub, sub_rhs,
                                                         [g["x"] for g in sub], axes=(0, 1, 2))
    except RuntimeError as e:  # device memory
        out["ir1_error"] = str(e)[:200]
    out["peak_GBps"] = peak()
    return out


def config4(rate=2000.0, seconds=2.0, n_problems=64, budget=150e9, seed=44):
    import torch

    import serving

    rng = np.random.default_rng(seed)
    shapes = [serving.log_uniform_dims(rng, 16, 512) for _ in range(n_problems)]
    pool = serving.ProblemPool(shapes, seed=seed)
    torch.cuda.synchronize()
    out = {"config": "config4_serving", "rate_per_s": rate, "pool_problems": n_problems,
           "pool_GB": round(pool.nbytes() / 1e9, 2), "budget_GB": budget / 1e9}
    n_req = int(rate * seconds)
    # untimed warm-up of every policy: first launches of each kernel variant
    # (module loading) and first plans happen here, not in the timed traces
    warm = serving.make_trace(256, math.inf, n_problems, seed=seed + 2)
    for policy in ("mixed", "fp64", "sequential"):
        serving.serve(pool, warm, policy, budget)
        torch.cuda.empty_cache()
    # the native serving handle's arena: the budget less the pool and the
    # requests' iterates, within what the device has free
    free, _ = torch.cuda.mem_get_info()
    arena = int(min(budget - pool.nbytes(), 0.4 * free))   # the rest: iterates, Python loop
    out["native_arena_GB"] = round(arena / 1e9, 2)
    for policy in ("mixed", "fp64", "sequential"):   # warm-up of the native path
        serving.serve_native(pool, warm, policy, arena)
        torch.cuda.empty_cache()
    for label, r in (("nominal", rate), ("saturated", math.inf)):
        # saturated: 8000 requests queued at t = 0 (about half a second of device work)
        trace = serving.make_trace(n_req if label == "nominal" else 2 * n_req, r, n_problems,
                                   seed=seed + 1)
        res = {}

        def fresh(run):
            # each implementation and policy first serves the trace untimed, from
            # empty iterate free lists, so the timed run meets its own steady state
            pool.drop_iterates()
            torch.cuda.empty_cache()
            run()

        for policy in ("mixed", "fp64", "sequential"):
            fresh(lambda: serving.serve(pool, trace, policy, budget))
            rep, ex, _ = serving.serve(pool, trace, policy, budget, calibrate=True)
            res[policy] = rep
            del ex
            fresh(lambda: serving.serve_native(pool, trace, policy, arena))
            rep, _, bits, _ = serving.serve_native(pool, trace, policy, arena, calibrate=True)
            rep["status_bits_nonzero"] = sum(1 for v in bits.values() if v)
            res[f"native_{policy}"] = rep
            torch.cuda.empty_cache()
        for pre in ("", "native_"):
            seq = res[f"{pre}sequential"]["solves_per_s"]
            res[f"{pre}speedup_mixed_vs_sequential"] = round(
                res[f"{pre}mixed"]["solves_per_s"] / seq, 3)
            res[f"{pre}speedup_fp64_vs_sequential"] = round(
                res[f"{pre}fp64"]["solves_per_s"] / seq, 3)
        out[label] = res
    return out


def config3_split(n_grids=96, lo=32, hi=384, seed=33):
    """Config 3's FP64 plans broken down: per axis, one plan per bucket of line
    length along that axis (n <= 256: du2 and dw2 in Tensor Memory; n > 256:
    dw2 with x2 through the buffer)."""
    import torch

    import pentadsolver as ps

    rng = np.random.default_rng(seed)
    dims_list = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(n_grids)]
    grids = [dev_problem(d, 1000 + i) for i, d in enumerate(dims_list)]
    out = {"config": "config3_split", "grids": n_grids, "seed": seed, "rows": []}
    buckets = ((32, 64), (65, 128), (129, 192), (193, 256), (257, 320), (321, 384))
    for axis in range(3):
        for b0, b1 in buckets + ((lo, hi),):
            idx = [i for i in range(n_grids) if b0 <= dims_list[i][axis] <= b1]
            if not idx:
                continue
            pts = sum(math.prod(dims_list[i]) for i in idx)
            with ps.Plan([grids[i] for i in idx], axis) as pl:
                ms = timed(lambda: pl.execute(), reps=5, warmup=2)
            out["rows"].append({"axis": axis, "n": [b0, b1], "grids": len(idx),
                                "Mpts": round(pts / 1e6, 1), "ms": round(ms, 3),
                                "GBps": round(56 * pts / ms / 1e6, 1)})
            torch.cuda.synchronize()
    out["peak_GBps"] = peak()
    return out


def config_refine1(n=512, calls=3):
    """One-step refined solves of config 2's grid (FP32 coefficient copies
    cached after the first call), `calls` timed calls per axis: the command
    whose kernel launch list shows where the refined form's time goes."""
    import pentadsolver as ps

    dims = (n, n, n)
    p = dev_problem(dims, 2)
    out = {"config": "refine1_512cube", "points": n ** 3, "axes": []}
    for axis in range(3):
        buf = ps.alloc_refine_buffer(list(dims), axis)
        args = (p["ds"], p["dl"], p["d"], p["du"], p["dw"], p["x"], axis)
        ps.gpsv_batch_refine(*args, steps=1, buffer=buf)
        ms = timed(lambda: ps.gpsv_batch_refine(*args, steps=1, buffer=buf,
                                                reuse_fp32_coefficients=True),
                   reps=calls, warmup=0)
        out["axes"].append({"axis": axis, "ms": round(ms, 4),
                            "GBps_equiv": round(56 * n ** 3 / ms / 1e6, 1)})
        del buf
    out["peak_GBps"] = peak()
    return out


def config_odd(reps=10):
    import os

    import torch

    import pentadsolver as ps

    out = {"config": "odd_sizes_single_solves", "rows": []}
    pk = peak()
    with ps.Handle() as h:
        for dtype in (torch.float64, torch.float32):
            eb = 8 if dtype == torch.float64 else 4
            for edge in (256, 255):
                dims = (edge, edge, edge)
                p = dev_problem(dims, 7, dtype)
                b = p["x"].clone()
                for loads in ("", "element", "group"):
                    if loads and edge % (16 // eb) == 0:
                        continue   # aligned: TMA tiles either way
                    os.environ["PENTA_TMEM_LOADS"] = loads
                    for axis in range(3):
                        buf = ps.alloc_buffer(list(dims), axis, dtype)

                        def run():
                            ps.gpsv_batch(p["ds"], p["dl"], p["d"], p["du"], p["dw"], p["x"],
                                          axis, buffer=buf, handle=h)

                        ms = timed(run, reps=reps, warmup=2)
                        p["x"].copy_(b)
                        d = 0 if axis == 0 else (2 if axis == 2 else 1)
                        gbs = 7 * eb * edge ** 3 / (ms * 1e-3) / 1e9
                        out["rows"].append({"dtype": "f64" if eb == 8 else "f32", "edge": edge,
                                            "axis": axis, "loads": loads or "default",
                                            "variant": h.variant_that_ran(d),
                                            "us": round(ms * 1e3, 1), "GBps": round(gbs, 1),
                                            "frac": round(gbs / pk, 3)})
                        del buf
                    os.environ.pop("PENTA_TMEM_LOADS", None)
                del p, b
                torch.cuda.empty_cache()
    # the 16 smallest grids of config 3 as FP64 plans (x, y, z), bulk and element loads
    rng = np.random.default_rng(33)
    dims_list = [tuple(int(v) for v in rng.integers(32, 385, size=3)) for _ in range(96)]
    sub = sorted(dims_list, key=math.prod)[:16]
    grids = [dev_problem(d, 500 + i) for i, d in enumerate(sub)]
    pts = sum(math.prod(d) for d in sub)
    for loads in ("", "element", "group"):
        os.environ["PENTA_TMEM_LOADS"] = loads
        plans = [ps.Plan(grids, axis) for axis in range(3)]
        ms = timed(lambda: [pl.execute() for pl in plans], reps=reps, warmup=2)
        out[f"subset16_plans_{loads or 'default'}"] = {
            "ms_xyz": round(ms, 3), "GBps": round(3 * 56 * pts / (ms * 1e-3) / 1e9, 1),
            "plans": [pl.describe() for pl in plans]}
        for pl in plans:
            pl.close()
        os.environ.pop("PENTA_TMEM_LOADS", None)
    del grids
    torch.cuda.empty_cache()
    # aligned 256^3 forced through the bulk-copy layout (against the TMA rows above)
    with ps.Handle() as h:
        for dtype in (torch.float64, torch.float32):
            eb = 8 if dtype == torch.float64 else 4
            dims = (256, 256, 256)
            p = dev_problem(dims, 7, dtype)
            os.environ["PENTA_TMEM_LOADS"] = "bulk"
            for axis in range(3):
                buf = ps.alloc_buffer(list(dims), axis, dtype)

                def run():
                    ps.gpsv_batch(p["ds"], p["dl"], p["d"], p["du"], p["dw"], p["x"], axis,
                                  buffer=buf, handle=h)

                ms = timed(run, reps=reps, warmup=2)
                d = 0 if axis == 0 else (2 if axis == 2 else 1)
                gbs = 7 * eb * 256 ** 3 / (ms * 1e-3) / 1e9
                out["rows"].append({"dtype": "f64" if eb == 8 else "f32", "edge": 256,
                                    "axis": axis, "loads": "bulk",
                                    "variant": h.variant_that_ran(d), "us": round(ms * 1e3, 1),
                                    "GBps": round(gbs, 1), "frac": round(gbs / pk, 3)})
                del buf
            os.environ.pop("PENTA_TMEM_LOADS", None)
            del p
            torch.cuda.empty_cache()
    out["peak_GBps"] = pk
    return out


def config_mesh(edge=256):
    import torch

    import mesh
    from oracle import oracle

    dims = (edge, edge, edge)
    solvedim = 2
    n_bytes = 6 * edge ** 3 * 8
    res = {"config": f"mesh_random_{edge}cube_fp64", "bytes": n_bytes,
           "host_threads": mesh.host_threads()}
    dev = {}
    for threads in sorted({mesh.host_threads(), 64, 148, 1024}):
        holder = {}

        def build():
            holder["m"] = mesh.random_mesh(dims, solvedim, threads, torch.float64)
        ms = timed(build, reps=3, warmup=1)
        dev[threads] = {"ms": round(ms, 3), "gbs": round(n_bytes / ms / 1e6, 1)}
        holder.clear()
    res["device_build"] = {str(k): v for k, v in dev.items()}
    if oracle.ref_mesh_available():
        t = mesh.host_threads()
        oracle.set_threads(t)
        t0 = time.time()
        ref = oracle.ref_mesh_random(dims, solvedim, t, np.float64)
        res["reference_host_build_ms"] = round((time.time() - t0) * 1e3, 1)
        torch.cuda.synchronize()
        t0 = time.time()
        up = {k: torch.from_numpy(ref[k]).to("cuda") for k in NAMES}
        torch.cuda.synchronize()
        res["reference_upload_ms"] = round((time.time() - t0) * 1e3, 1)
        got = mesh.random_mesh(dims, solvedim, t, torch.float64)
        torch.cuda.synchronize()
        res["bit_identical_to_reference"] = all(torch.equal(got[k].view(torch.int64),
                                                            up[k].view(torch.int64))
                                                for k in NAMES)
        res["reference_total_ms"] = round(res["reference_host_build_ms"] +
                                          res["reference_upload_ms"], 1)
        res["speedup_same_threads"] = round(res["reference_total_ms"] / dev[t]["ms"], 1)
    else:
        res["reference"] = "oracle/_ref/libmesh_ref.so not built"
    return res


def config_refapp(edge=256, iters=50):
    import os
    import subprocess

    ref_dir = REPO / "oracle" / "_ref"
    apps = {"reference": ref_dir / "app_cuda_ref", "b200": ref_dir / "app_cuda_b200"}
    missing = [str(v) for v in apps.values() if not v.exists()]
    if missing:
        return {"config": "refapp", "unavailable": f"not built: {missing}"}
    runs = [("double", {}), ("float", {}),
            ("double", {"PENTA_XALGO": "shared-fact", "PENTA_YZALGO": "shared-fact"})]
    out = {"config": f"reference_adi_app_{edge}cube", "iters": iters, "runs": []}
    for prec, env in runs:
        elem = 8 if prec == "double" else 4
        per_point = 2 * elem if env else 7 * elem  # shared factorisation: RHS in, x out
        alg = 3 * per_point * edge ** 3
        row = {"precision": prec, "selectors": env or "default"}
        for name, app in apps.items():
            e = dict(os.environ)
            e.update(env)
            r = subprocess.run([str(app), str(edge), str(iters), prec], env=e,
                               capture_output=True, text=True, timeout=300)
            csv_line = [ln for ln in r.stdout.splitlines() if ln.startswith("CSV,")]
            if r.returncode != 0 or not csv_line:
                row[name] = {"error": (r.stderr or r.stdout)[-300:]}
                continue
            f = csv_line[-1].split(",")
            ev_ms = float(f[10])
            row[name] = {"kernels": [f[2], f[4], f[6]], "iter_ms_wall": float(f[9]),
                         "iter_ms_events": ev_ms,
                         "per_direction_ms": [float(f[11]), float(f[12]), float(f[13])],
                         "gbs": round(alg / (ev_ms * 1e-3) / 1e9, 1)}
        if "iter_ms_events" in row.get("reference", {}) and \
                "iter_ms_events" in row.get("b200", {}):
            row["speedup"] = round(row["reference"]["iter_ms_events"] /
                                   row["b200"]["iter_ms_events"], 2)
        out["runs"].append(row)
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--configs", default="0,2,3,4")
    ap.add_argument("--n2", type=int, default=512, help="grid edge of config 2")
    ap.add_argument("--grids3", type=int, default=96)
    ap.add_argument("--seconds4", type=float, default=2.0)
    ap.add_argument("--odd-reps", type=int, default=10, help="timed solves per case (odd)")
    args = ap.parse_args()
    want = {c.strip() for c in args.configs.split(",")}
    runs = {"0": config0, "2": lambda: config2(args.n2), "3": lambda: config3(args.grids3),
            "4": lambda: config4(seconds=args.seconds4), "mesh": config_mesh,
            "refapp": config_refapp, "odd": lambda: config_odd(args.odd_reps),
            "3split": config3_split, "refine1": config_refine1}
    from bench import ClockSampler

    for c in ("0", "2", "refine1", "3", "3split", "4", "odd", "mesh", "refapp"):
        if c in want:
            t0 = time.time()
            with ClockSampler(0) as clk:
                res = runs[c]()
            res["clocks"] = clk.summary()
            res["wall_s"] = round(time.time() - t0, 1)
            print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
