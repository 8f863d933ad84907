"""Parity at the shapes of the precision, batched and serving workloads.

Every result is compared with the CPU oracle (``oracle/penta_oracle.c``, the
restatement of ``src/cpu/singlenode/pentad_orig_cpu.cpp``), never with another
GPU result.  Forward error is the one the reference's accuracy app uses,
``max|x - x_ref| / max|x_ref|`` over the grid (``apps/fp32_accuracy_cuda.cu:
326-343``); tolerances: plain FP64 1e-12, FP32 sweeps + FP64 refinement 1e-10.

* Precision form (512^3 random dominant grids): lines of n = 512 along each
  axis -- the factor mode the 512^3 grid takes (dw2 through the buffer in
  FP64) -- with a small cross-section so the oracle finishes in a second;
  plain FP64, and FP32 sweeps with 1, 2 and 3 refinement steps.
* Batched uneven grids (96 grids, N ~ U[32,384], seed 33): the 16 smallest
  grids of that seeded list (odd and even extents, up to 359), as FP64 plans
  for x, y and z captured together in one CUDA graph and replayed, and as
  refinement plans per axis.
* Serving (Poisson stream, N ~ logU[16,512] per axis, solvedim U{0,1,2}, 70%
  at tolerance 1e-10 and 30% at 1e-13): every served result of the mixed and
  FP64 policies against the oracle, at the request's own tolerance.
"""
from __future__ import annotations

import math
import os

import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
REFINED_TOL = 1e-10


@pytest.fixture(scope="module", autouse=True)
def _oracle_threads():
    oracle.set_threads(os.cpu_count() or 1)


def oracle_solution(co: dict, solvedim: int) -> np.ndarray:
    x = co["x"].copy()
    oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x, solvedim)
    return x


# ---------------------------------------------------------------- precision
@pytest.mark.parametrize("solvedim, dims", [(0, (512, 40, 36)), (1, (40, 512, 36)),
                                            (2, (36, 40, 512))])
def test_precision_form_n512_against_the_oracle(cuda, solvedim, dims):
    import torch

    co = fixtures.random_dominant(dims, 512 + solvedim, np.float64)
    ref = oracle_solution(co, solvedim)
    with ps.Handle() as h:
        dv = to_dev(co)
        buf = ps.alloc_buffer(list(dims), solvedim, torch.float64)
        ps.gpsv_batch(*(dv[k] for k in NAMES), solvedim, buffer=buf, handle=h)
        torch.cuda.synchronize()
        assert " w2s" in h.variant_that_ran(0 if solvedim == 0 else (2 if solvedim == 2 else 1))
        assert fwd_err(dv["x"].cpu().numpy(), ref) <= FP64_TOL
        rbuf = ps.alloc_refine_buffer(list(dims), solvedim)
        errs = []
        for steps in range(4):
            dv = to_dev(co)
            ps.gpsv_batch_refine(*(dv[k] for k in NAMES), solvedim, steps=steps, buffer=rbuf,
                                 handle=h)
            torch.cuda.synchronize()
            errs.append(fwd_err(dv["x"].cpu().numpy(), ref))
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
    assert errs[0] > 1e-9, errs                 # the FP32 sweep alone is not enough
    assert max(errs[1:]) <= REFINED_TOL, errs   # one step reaches the tolerance


# ------------------------------------------------------------------ batched
def batched_subset(count=16, seed=33, lo=32, hi=384, n_grids=96):
    """The `count` smallest grids of the seeded 96-grid list."""
    rng = np.random.default_rng(seed)
    dims_list = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(n_grids)]
    order = sorted(range(n_grids), key=lambda i: math.prod(dims_list[i]))
    return [(i, dims_list[i]) for i in sorted(order[:count])]


def test_batched_subset_keeps_the_workloads_extents():
    sub = batched_subset()
    ext = [v for _, d in sub for v in d]
    assert len(sub) == 16 and max(ext) >= 350 and min(ext) >= 32
    assert any(v % 2 for v in ext) and any(v % 2 == 0 for v in ext)


def test_batched_uneven_grids_fp64_graph_against_the_oracle(cuda):
    import torch

    sub = batched_subset()
    probs = [fixtures.random_dominant(d, 1000 + i, np.float64) for i, d in sub]
    refs = []
    for co in probs:
        x = co["x"].copy()
        for axis in range(3):   # x, then y, then z on the result, as the workload runs
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x, axis)
        refs.append(x)
    devs = [to_dev(co) for co in probs]
    rhs = [dv["x"].clone() for dv in devs]
    shared = ps.aligned_bytes(max(ps.plan_sizes(devs, a)[1] for a in range(3)))
    plans = [ps.Plan(devs, axis, scratch=shared) for axis in range(3)]
    try:
        s = torch.cuda.Stream()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            for pl in plans:
                pl.execute(s)
        for dv, r in zip(devs, rhs):
            dv["x"].copy_(r)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        for (i, dims), dv, ref in zip(sub, devs, refs):
            e = fwd_err(dv["x"].cpu().numpy(), ref)
            assert e <= FP64_TOL, (i, dims, e)
        for pl in plans:
            assert pl.status_check() == (ps.SUCCESS, 0), pl.describe()
        del graph
    finally:
        for pl in plans:
            pl.close()


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_batched_uneven_grids_refined_against_the_oracle(cuda, solvedim):
    sub = batched_subset()
    probs = [fixtures.random_dominant(d, 1000 + i, np.float64) for i, d in sub]
    refs = [oracle_solution(co, solvedim) for co in probs]
    devs = [to_dev(co) for co in probs]
    with ps.Plan(devs, solvedim, refine_steps=1) as plan:
        plan.execute()
        est = plan.estimates()
        assert plan.status_check() == (ps.SUCCESS, 0)
    for (i, dims), dv, ref, (dmax, xmax) in zip(sub, devs, refs, est):
        e = fwd_err(dv["x"].cpu().numpy(), ref)
        assert e <= REFINED_TOL, (i, dims, solvedim, e)
        assert xmax > 0 and dmax / xmax < 1e-5, (i, dims, dmax, xmax)


# ------------------------------------------------------------------ serving
@pytest.mark.parametrize("policy", ["mixed", "fp64"])
def test_served_results_against_the_oracle(cuda, policy):
    import serving

    rng = np.random.default_rng(44)
    shapes = []
    while len(shapes) < 12:   # N ~ logU[16, 512] per axis; volumes the oracle takes fast
        d = serving.log_uniform_dims(rng, 16, 512)
        if math.prod(d) <= 2_000_000:
            shapes.append(d)
    assert max(max(d) for d in shapes) >= 256
    pool = serving.ProblemPool(shapes, seed=45)
    trace = serving.make_trace(60, math.inf, len(shapes), seed=46)
    assert {r.solvedim for r in trace} == {0, 1, 2}
    assert {r.tol for r in trace} == {1e-10, 1e-13}
    rep, ex, tr = serving.serve(pool, trace, policy, budget_bytes=8e9, max_batch=16,
                                keep_results=True)
    assert rep["requests"] == 60
    host = [{k: v.cpu().numpy() for k, v in p.items()} for p in pool.items]
    refs = {}
    for r in tr:
        key = (r.problem, r.solvedim)
        if key not in refs:
            p = host[r.problem]
            x = p["b"].copy()
            oracle.solve(p["ds"], p["dl"], p["d"], p["du"], p["dw"], x, r.solvedim)
            refs[key] = x
        got = ex.results[r.rid].cpu().numpy()
        e = fwd_err(got, refs[key])
        tol = REFINED_TOL if (policy == "mixed" and r.tol >= 1e-10) else FP64_TOL
        assert e <= tol, (r.rid, shapes[r.problem], r.solvedim, r.tol, e)
    assert not any(ex.status.values())
