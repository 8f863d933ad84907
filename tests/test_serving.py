"""Host logic of the serving loop (pentadiagonal-solver_b200/serving.py) on
CPU: the Poisson trace, admission by HBM budget, continuous batching by
(solvedim, precision class), the sequential baseline, and the latency
report -- driven by a fake executor on a simulated clock."""
import math

import numpy as np
import pytest

import serving


class FakeExecutor:
    """Simulated GPU: a batch takes 20 us + 1 ns per point; up to three run
    at once; the clock only advances when the scheduler idles."""

    def __init__(self, points):
        self.points = points
        self.t = 0.0
        self.log = []

    def now(self):
        return self.t

    def idle(self, until=None):
        self.t = max(self.t + 1e-6, until if until is not None else 0.0)

    def request_bytes(self, r):
        return 8 * self.points[r.problem]

    def batch_bytes(self, reqs, key):
        return sum(24 * self.points[r.problem] for r in reqs)

    def launch(self, b):
        cost = 20e-6 + 1e-9 * sum(self.points[r.problem] for r in b.requests)
        self.log.append((b.key, [r.rid for r in b.requests], self.t))
        return self.t + cost

    def done(self, token):
        return self.t >= token

    def finish(self, b):
        pass


def test_trace_is_poisson_with_the_stated_mix():
    tr = serving.make_trace(4000, 2000.0, 16, seed=1)
    gaps = np.diff([r.arrival for r in tr])
    assert abs(gaps.mean() - 1 / 2000.0) < 0.05 / 2000.0
    assert all(r.solvedim in (0, 1, 2) for r in tr)
    loose = sum(r.tol == 1e-10 for r in tr) / len(tr)
    assert 0.67 < loose < 0.73
    burst = serving.make_trace(10, math.inf, 4, seed=2)
    assert all(r.arrival == 0.0 for r in burst)


@pytest.mark.parametrize("policy", ["mixed", "fp64", "sequential"])
def test_scheduler_completes_everything_within_budget(policy):
    rng = np.random.default_rng(3)
    points = [int(v) for v in rng.integers(1000, 200000, size=12)]
    ex = FakeExecutor(points)
    budget = 40e6
    sch = serving.Scheduler(ex, budget, max_batch=8,
                            max_in_flight=1 if policy == "sequential" else 3, policy=policy)
    tr = serving.make_trace(300, 20000.0, len(points), seed=4)
    sch.run(tr)
    assert all(math.isfinite(r.done) and r.done >= r.started >= r.admitted >= r.arrival
               for r in tr)
    assert sch.peak <= budget
    keys = [k for k, _, _ in ex.log]
    if policy == "sequential":
        assert all(len(ids) == 1 for _, ids, _ in ex.log)
    else:
        for key, ids, _ in ex.log:
            reqs = [tr[i] for i in ids]
            assert len(ids) <= 8
            assert all(r.solvedim == key[0] for r in reqs)
            if key[1] == "f64" and policy == "mixed":
                assert all(not r.mixed_ok for r in reqs)
            if policy == "fp64":
                assert key[1] == "f64"
        assert len(ex.log) < len(tr)       # requests were batched
    rep = serving.report(tr)
    assert rep["requests"] == 300 and rep["p99_ms"] >= rep["p50_ms"] > 0


def test_admission_waits_for_memory_and_keeps_arrival_order():
    points = [1_000_000] * 4
    ex = FakeExecutor(points)
    # room for one request and its scratch at a time
    sch = serving.Scheduler(ex, 8e6 + 24e6, max_batch=4, policy="fp64")
    tr = serving.make_trace(12, math.inf, 4, seed=5)
    sch.run(tr)
    starts = [r.started for r in sorted(tr, key=lambda r: r.rid)]
    assert starts == sorted(starts)
    assert sch.peak <= 8e6 + 24e6
    assert all(len(ids) == 1 for _, ids, _ in ex.log)


def test_mixed_policy_routes_loose_requests_by_measured_cost():
    # an executor that measured refinement slower along y only: loose y
    # requests then join the FP64 batches, the others stay mixed
    class Costed(FakeExecutor):
        def refine_pays(self, solvedim):
            return solvedim != 1

    ex = Costed([1000] * 4)
    sch = serving.Scheduler(ex, 1e12, policy="mixed")
    loose = [serving.Request(i, 0.0, 0, d, 1e-10) for i, d in enumerate((0, 1, 2))]
    tight = serving.Request(9, 0.0, 0, 1, 1e-13)
    assert [sch.key_of(r) for r in loose] == [(0, "mixed"), (1, "f64"), (2, "mixed")]
    assert sch.key_of(tight) == (1, "f64")
    # without a measurement the loose requests are mixed
    plain = serving.Scheduler(FakeExecutor([1000]), 1e12, policy="mixed")
    assert plain.key_of(loose[1]) == (1, "mixed")


def test_native_server_refuses_bad_arguments_before_touching_a_device():
    import ctypes

    import pentadsolver as ps

    f = ps._typed("pentadsolver_server_create",
                  [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int, ctypes.c_int,
                   ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)])
    out = ctypes.c_void_p(None)
    good = dict(arena=1 << 20, nbytes=1 << 20, policy=0, streams=3, batch=8, inflight=3, steps=1)
    for bad in ({"arena": 0}, {"arena": (1 << 20) + 8}, {"nbytes": 100}, {"policy": 3},
                {"streams": 0}, {"batch": 0}, {"inflight": 0}, {"steps": 9}):
        a = {**good, **bad}
        st = f(None, a["arena"], a["nbytes"], a["policy"], a["streams"], a["batch"],
               a["inflight"], a["steps"], ctypes.byref(out))
        assert st == ps.INVALID_VALUE and not out.value, bad
