"""The library's serving handle (pentadsolver_server_*) on the GPU.

A config-4-shaped stream (per-axis N ~ logU[16,512], solvedim U{0,1,2}, 70% at
tolerance 1e-10, 30% at 1e-13) is replayed through the native handle under
each policy: every result equals the oracle's at its request's tolerance,
every batch reports a clean status word, continuous batching forms fewer
batches than requests (one per request for the sequential baseline), and the
batch memory never exceeds the arena -- also when the arena is too small for
everything at once.  A request larger than the whole arena is rejected, not
stalled.
"""
import math

import numpy as np
import pytest

import pentadsolver as ps
import serving
from gpu_util import fwd_err
from oracle import oracle

pytestmark = pytest.mark.gpu


def _pool(seed=44, count=12, cap=2_000_000):
    rng = np.random.default_rng(seed)
    shapes = []
    while len(shapes) < count:
        d = serving.log_uniform_dims(rng, 16, 512)
        if math.prod(d) <= cap:
            shapes.append(d)
    return serving.ProblemPool(shapes, seed=seed + 1)


def _oracle_refs(pool, trace):
    host = [{k: v.cpu().numpy() for k, v in p.items()} for p in pool.items]
    refs = {}
    for r in trace:
        key = (r.problem, r.solvedim)
        if key not in refs:
            p = host[r.problem]
            x = p["b"].copy()
            oracle.solve(p["ds"], p["dl"], p["d"], p["du"], p["dw"], x, r.solvedim)
            refs[key] = x
    return refs


@pytest.mark.parametrize("policy,calibrate", [("mixed", True), ("mixed", False),
                                              ("fp64", True), ("sequential", True)])
def test_native_server_results_against_the_oracle(cuda, policy, calibrate):
    # uncalibrated, the mixed policy refines every loose request (FP32 sweeps +
    # FP64 refinement); calibrated on B200 it measures refinement slower and
    # serves them in FP64
    pool = _pool()
    trace = serving.make_trace(60, math.inf, len(pool.shapes), seed=46)
    rep, results, bits, tr = serving.serve_native(pool, trace, policy, arena_bytes=4e9,
                                                  max_batch=16, keep_results=True,
                                                  calibrate=calibrate)
    assert rep["requests"] == 60 and len(results) == 60
    if policy == "sequential":
        assert rep["batches"] == 60
    else:
        assert rep["batches"] < 60
    assert rep["peak_arena_gb"] <= 4.0
    assert rep["p99_ms"] >= rep["p50_ms"] > 0
    assert not any(bits.values())
    refs = _oracle_refs(pool, tr)
    for r in tr:
        e = fwd_err(results[r.rid].cpu().numpy(), refs[(r.problem, r.solvedim)])
        tol = 1e-10 if (policy == "mixed" and r.tol >= 1e-10) else 1e-12
        assert e <= tol, (r.rid, pool.shapes[r.problem], r.solvedim, r.tol, e)


def test_native_server_respects_a_small_arena(cuda):
    import torch

    pool = _pool(seed=50, count=6, cap=400_000)
    arena = 24 * 1024 * 1024
    srv = serving.NativeServer(arena, "fp64", max_batch=64)
    xs = {}
    for i in range(40):
        pi = i % len(pool.shapes)
        p = pool.items[pi]
        x = p["b"].clone()
        rid = srv.submit({**{k: p[k] for k in ("ds", "dl", "d", "du", "dw")}, "x": x},
                         i % 3, 1e-13)
        xs[rid] = (pi, i % 3, x)
    torch.cuda.synchronize()   # the iterates' copies, before the server's streams read them
    srv.progress(wait=True)
    done = dict(srv.poll())
    st = srv.stats()
    srv.close()
    torch.cuda.synchronize()
    assert sorted(done) == sorted(xs) and not any(done.values())
    assert st["arena_peak"] <= arena and st["batches"] > 1 and st["queued"] == 0
    host = [{k: v.cpu().numpy() for k, v in p.items()} for p in pool.items]
    for rid, (pi, sd, x) in xs.items():
        p = host[pi]
        ref = p["b"].copy()
        oracle.solve(p["ds"], p["dl"], p["d"], p["du"], p["dw"], ref, sd)
        assert fwd_err(x.cpu().numpy(), ref) <= 1e-12


def test_native_server_rejects_a_request_larger_than_its_arena(cuda):
    import torch

    # lines of 256 along x: x2 goes through the plan's scratch (16 MB here);
    # lines of at most 160 would keep everything in Tensor Memory and fit
    pool = serving.ProblemPool([(256, 128, 64)], seed=51)
    srv = serving.NativeServer(1 << 20, "fp64")   # 1 MiB: the grid's plan cannot fit
    p = pool.items[0]
    rid = srv.submit({**{k: p[k] for k in ("ds", "dl", "d", "du", "dw")}, "x": p["b"].clone()},
                     0, 1e-13)
    torch.cuda.synchronize()
    srv.progress(wait=True)
    assert srv.poll() == [(rid, 1 << 30)]   # PENTADSOLVER_SERVER_REJECTED_BIT
    srv.close()
