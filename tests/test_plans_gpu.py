"""GPU parity of plans (many uneven grids in one persistent launch, CUDA-graph
capture) and of mixed-precision refinement (FP32 sweeps, FP64 residual and
correction).

Tolerances: plain plans as single solves (forward error <= 1e-12 FP64,
<= 1e-5 FP32 against the oracle); refinement <= 1e-10 against the FP64
oracle after one or more refinement steps (the precision form's target).
"""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, solve_dev, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

FWD_TOL = {np.float64: 1e-12, np.float32: 1e-5}


def uneven_dims(count, seed, lo=5, hi=60, extra=()):
    rng = np.random.default_rng(seed)
    out = [tuple(int(v) for v in rng.integers(lo, hi + 1, size=3)) for _ in range(count)]
    return out + list(extra)


def oracle_solution(co, solvedim):
    ref = {k: co[k].astype(np.float64) for k in NAMES}
    oracle.solve(ref["ds"], ref["dl"], ref["d"], ref["du"], ref["dw"], ref["x"], solvedim)
    return ref["x"]


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_plan_uneven_grids_match_oracle(cuda, dtype, solvedim):
    # odd and even extents, lines of 5 (solved alone: too short for the halves
    # of the batched kernel), and long lines (du2-only factor mode)
    extra = [(300, 6, 5), (6, 290, 5), (5, 5, 260), (5, 5, 5), (64, 64, 64), (1040, 16, 5),
             (5, 16, 1100)]
    dims_list = uneven_dims(14, 100 + solvedim, extra=extra)
    probs = [fixtures.random_dominant(dims, 40 + i, dtype) for i, dims in enumerate(dims_list)]
    refs = [oracle_solution(co, solvedim) for co in probs]
    devs = [to_dev(co) for co in probs]
    with ps.Plan(devs, solvedim) as plan:
        desc = plan.describe()
        plan.execute()
        st, bits = plan.status_check()   # the plan's own status word
        assert st == ps.SUCCESS and bits == 0, desc
    assert "tmem-batch" in desc, desc
    for dims, dv, ref in zip(dims_list, devs, refs):
        e = fwd_err(dv["x"].cpu().numpy(), ref)
        assert e <= FWD_TOL[dtype], (dims, solvedim, e, desc)


def test_plan_graph_capture_and_replay(cuda):
    """x, y and z plans captured into one CUDA graph; replays on fresh
    right-hand sides give the same bits as eager executes."""
    import torch

    dims_list = uneven_dims(10, 7, lo=8, hi=48)
    probs = [fixtures.random_dominant(dims, 70 + i, np.float64) for i, dims in enumerate(dims_list)]
    devs = [to_dev(co) for co in probs]
    rhs0 = [dv["x"].clone() for dv in devs]
    # the three plans share one scratch region (they never run at once)
    shared = ps.aligned_bytes(max(ps.plan_sizes(devs, a)[1] for a in range(3)))
    plans = [ps.Plan(devs, axis, scratch=shared) for axis in range(3)]
    # eager reference
    for p in plans:
        p.execute()
    torch.cuda.synchronize()
    eager = [dv["x"].clone() for dv in devs]
    # capture
    stream = torch.cuda.Stream()
    for dv, r in zip(devs, rhs0):
        dv["x"].copy_(r)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        for p in plans:
            p.execute(stream)
    for _ in range(2):
        for dv, r in zip(devs, rhs0):
            dv["x"].copy_(r)
        graph.replay()
        torch.cuda.synchronize()
        for dv, e in zip(devs, eager):
            assert torch.equal(dv["x"], e)
    # and against the oracle
    for co, dv in zip(probs, devs):
        ref = co["x"].copy()
        for axis in range(3):
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
        assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12
    del graph
    for p in plans:
        p.close()


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_refine_reaches_the_fp64_tolerance(cuda, solvedim):
    """FP32 sweeps alone miss 1e-10 by orders of magnitude; one refinement
    step reaches it; more steps do not get worse; the estimate tracks it."""
    dims = (48, 40, 36)
    co = fixtures.random_dominant(dims, 5 + solvedim, np.float64)
    ref = oracle_solution(co, solvedim)
    errs = []
    for steps in range(4):
        dv = to_dev(co)
        buf = ps.alloc_refine_buffer(list(dims), solvedim)
        ps.gpsv_batch_refine(*(dv[k] for k in NAMES), solvedim, steps=steps, buffer=buf)
        errs.append(fwd_err(dv["x"].cpu().numpy(), ref))
        if steps >= 1:
            dmax, xmax = ps.refine_estimate(buf)
            assert 0 < xmax and dmax / xmax < 1e-4
    assert errs[0] > 1e-9, errs          # FP32 sweep alone
    assert max(errs[1:]) <= 1e-10, errs  # refined
    assert ps.status_check()[1] == 0


@pytest.mark.parametrize("steps", [1, 2])   # the one-step form and the general one
def test_refine_reuses_fp32_coefficients(cuda, steps):
    dims = (40, 32, 24)
    co = fixtures.random_dominant(dims, 9, np.float64)
    ref = oracle_solution(co, 1)
    dv = to_dev(co)
    buf = ps.alloc_refine_buffer(list(dims), 1)
    ps.gpsv_batch_refine(*(dv[k] for k in NAMES), 1, steps=steps, buffer=buf)
    first = dv["x"].clone()
    dv["x"].copy_(to_dev(co)["x"])
    ps.gpsv_batch_refine(*(dv[k] for k in NAMES), 1, steps=steps, buffer=buf,
                         reuse_fp32_coefficients=True)
    import torch

    assert torch.equal(dv["x"], first)
    assert fwd_err(first.cpu().numpy(), ref) <= 1e-10


def test_refine_one_step_same_bits_on_unaligned_arrays(cuda):
    # arrays one element past a 16-byte boundary take the element-wise FP64
    # steps one point at a time instead of in pairs: the same bits
    import torch

    dims = (37, 30, 22)
    co = fixtures.random_dominant(dims, 13, np.float64)
    n = int(np.prod(dims))
    results = []
    for shift in (0, 1):
        dv = {}
        for k in NAMES:
            raw = torch.empty(n + 2, dtype=torch.float64, device="cuda")
            dv[k] = raw[shift:shift + n].view(*reversed(dims))
            dv[k].copy_(torch.from_numpy(co[k]))
        assert (dv["x"].data_ptr() % 16 == 0) == (shift == 0)
        buf = ps.alloc_refine_buffer(list(dims), 0)
        ps.gpsv_batch_refine(*(dv[k] for k in NAMES), 0, steps=1, buffer=buf)
        results.append((dv["x"].clone(), ps.refine_estimate(buf)))
    assert torch.equal(results[0][0], results[1][0])
    assert results[0][1] == results[1][1]
    ref = oracle_solution(co, 0)
    assert fwd_err(results[0][0].cpu().numpy(), ref) <= 1e-10


@pytest.mark.parametrize("steps", [1, 2])
def test_refine_plan_reuses_its_fp32_copies(cuda, steps):
    # an execute that keeps the FP32 copies of an earlier execute gives the same
    # bits as one that casts again; the first execute casts even when asked to
    # reuse
    import torch

    dims_list = [(33, 20, 17), (48, 24, 12)]
    probs = [fixtures.random_dominant(d, 70 + i, np.float64) for i, d in enumerate(dims_list)]
    devs = [to_dev(co) for co in probs]
    rhs = [dv["x"].clone() for dv in devs]
    with ps.Plan(devs, 1, refine_steps=steps) as plan:
        plan.execute(reuse_fp32=True)
        first = [dv["x"].clone() for dv in devs]
        for dv, r in zip(devs, rhs):
            dv["x"].copy_(r)
        plan.execute(reuse_fp32=True)
        again = [dv["x"].clone() for dv in devs]
        assert plan.status_check() == (ps.SUCCESS, 0)
    for a, b, co in zip(first, again, probs):
        assert torch.equal(a, b)
        assert fwd_err(a.cpu().numpy(), oracle_solution(co, 1)) <= 1e-10


def test_refine_estimate_reads_zero_without_a_step(cuda):
    # the estimate slot of a buffer that held anything reads (0, 0) after a
    # solve without refinement steps
    dims = (32, 24, 20)
    co = fixtures.random_dominant(dims, 12, np.float64)
    dv = to_dev(co)
    buf = ps.alloc_refine_buffer(list(dims), 2)
    buf.fill_(0x7F)
    ps.gpsv_batch_refine(*(dv[k] for k in NAMES), 2, steps=0, buffer=buf)
    assert ps.refine_estimate(buf) == (0.0, 0.0)


@pytest.mark.parametrize("steps", [1, 2])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_refine_plan_uneven_grids(cuda, solvedim, steps):
    dims_list = uneven_dims(10, 300 + solvedim, lo=6, hi=50, extra=[(300, 5, 6)])
    probs = [fixtures.random_dominant(dims, 90 + i, np.float64) for i, dims in enumerate(dims_list)]
    refs = [oracle_solution(co, solvedim) for co in probs]
    devs = [to_dev(co) for co in probs]
    with ps.Plan(devs, solvedim, refine_steps=steps) as plan:
        plan.execute()
        est = plan.estimates()
        desc = plan.describe()
        assert plan.status_check() == (ps.SUCCESS, 0)
    assert f"refine steps={steps}" in desc
    for dims, dv, ref, (dmax, xmax) in zip(dims_list, devs, refs, est):
        e = fwd_err(dv["x"].cpu().numpy(), ref)
        assert e <= 1e-10, (dims, solvedim, e)
        # the last correction's size: the FP32 iterate's error after one step
        assert xmax > 0 and dmax / xmax < (1e-4 if steps == 1 else 1e-6), (dims, dmax, xmax)
    assert ps.status_check()[1] == 0
