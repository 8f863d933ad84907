"""The served mixed-size stream on the GPU: every result equals the same
request solved alone by a plain FP64 call, within the request's tolerance
(1e-10 for mixed-precision requests, 1e-12 for FP64 ones), whatever else
shared its batch; and the loop reports latency percentiles."""
import math

import numpy as np
import pytest

import pentadsolver as ps
import serving
from gpu_util import fwd_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("policy", ["mixed", "fp64"])
def test_each_result_is_the_same_alone_and_in_the_mix(cuda, policy):
    import torch

    rng = np.random.default_rng(11)
    shapes = [serving.log_uniform_dims(rng, 16, 72) for _ in range(10)]
    pool = serving.ProblemPool(shapes, seed=3)
    trace = serving.make_trace(48, 4000.0, len(shapes), seed=12)
    rep, ex, tr = serving.serve(pool, trace, policy, budget_bytes=4e9, max_batch=16,
                                keep_results=True)
    assert rep["requests"] == 48 and rep["batches"] < 48
    assert rep["p99_ms"] >= rep["p50_ms"] > 0
    for r in tr:
        p = pool.items[r.problem]
        x = p["b"].clone()
        buf = ps.alloc_buffer(ps.dims_of(x), r.solvedim, torch.float64)
        ps.gpsv_batch(p["ds"], p["dl"], p["d"], p["du"], p["dw"], x, r.solvedim, buffer=buf)
        torch.cuda.synchronize()
        got = ex.results[r.rid].cpu().numpy()
        e = fwd_err(got, x.cpu().numpy())
        tol = 1e-10 if (policy == "mixed" and r.tol >= 1e-10) else 1e-12
        assert e <= tol, (r.rid, shapes[r.problem], r.solvedim, r.tol, e)
    # every request's batch reported a clean status word of its own
    assert sorted(ex.status) == sorted(r.rid for r in tr)
    assert not any(ex.status.values())
    assert ps.status_check()[1] == 0


def test_sequential_baseline_runs_one_call_at_a_time(cuda):
    rng = np.random.default_rng(13)
    shapes = [serving.log_uniform_dims(rng, 16, 48) for _ in range(4)]
    pool = serving.ProblemPool(shapes, seed=4)
    trace = serving.make_trace(12, math.inf, len(shapes), seed=14)
    rep, ex, tr = serving.serve(pool, trace, "sequential", budget_bytes=4e9)
    assert rep["batches"] == 12
    done = sorted(r.done for r in tr)
    starts = sorted(r.started for r in tr)
    assert all(s >= d for s, d in zip(starts[1:], done[:-1]))
