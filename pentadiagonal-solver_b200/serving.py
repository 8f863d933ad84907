"""Serving: a continuous-batching request loop over device-resident problems.

Requests (a grid shape, a solve direction, a tolerance) arrive on a clock --
a Poisson stream in the benchmarks.  The loop

  * admits queued requests first come, first served while their device
    memory (the request's iterate plus the scratch of the plan that will
    solve it) fits the HBM budget;
  * groups admitted requests by (solvedim, precision class) and launches each
    group as one plan -- one persistent launch for all its grids -- on one of
    several CUDA streams, so batches overlap on the device and requests that
    arrive while others run join the next batch as soon as memory frees;
  * keeps coefficients device-resident (a pool of problems built once) and
    each request's iterate on the device from admission to completion;
  * records each request's latency (completion minus arrival) and reports
    p50/p99 beside throughput.

Precision classes: requests at tolerance >= 1e-10 may use mixed precision
(FP32 sweeps + FP64 refinement) under the "mixed" policy; tighter ones always
use plain FP64.  The mixed policy takes the refined form only where it pays:
the executor measures, per solve direction, a refinement plan against a
plain FP64 plan on the pool's largest problem at start-up, and loose
requests of a direction whose refined form measured slower run in FP64.  (On
a part whose FP64 sweep is bandwidth-bound, as on B200, that is every
direction: the refined form moves more bytes per point than plain FP64.)  The "sequential" policy is the baseline: each request solved
alone by one plain FP64 call, in arrival order.

The scheduler (admission, grouping, budget accounting) is independent of the
GPU: ``Scheduler`` drives an executor object, and the CUDA executor here is
one implementation of it.
"""
from __future__ import annotations

import contextlib
import gc
import math
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float          # seconds from the start of the trace
    problem: int            # index into the problem pool
    solvedim: int
    tol: float
    admitted: float = math.nan
    started: float = math.nan
    done: float = math.nan
    batch: int = -1

    @property
    def mixed_ok(self) -> bool:
        return self.tol >= 1e-10


def log_uniform_dims(rng, lo, hi, ndim=3):
    return tuple(int(round(math.exp(rng.uniform(math.log(lo), math.log(hi))))) for _ in range(ndim))


def make_trace(n_requests: int, rate: float, n_problems: int, seed: int,
               frac_loose: float = 0.7) -> list[Request]:
    """Poisson arrivals (exponential gaps, mean 1/rate; rate = inf puts every
    request at t = 0), uniform problem index, solvedim U{0,1,2}, tolerance
    1e-10 with probability frac_loose, else 1e-13."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        if math.isfinite(rate):
            t += rng.exponential(1.0 / rate)
        out.append(Request(i, t, int(rng.integers(n_problems)), int(rng.integers(3)),
                           1e-10 if rng.random() < frac_loose else 1e-13))
    return out


@contextlib.contextmanager
def no_gc():
    """Python's cyclic garbage collector paused while a trace is served, so
    that its pauses do not land in the latencies (it runs once afterwards)."""
    enabled = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if enabled:
            gc.enable()
        gc.collect()


def percentile(values, q):
    v = sorted(values)
    if not v:
        return math.nan
    k = (len(v) - 1) * q
    lo, hi = math.floor(k), math.ceil(k)
    return v[lo] + (v[hi] - v[lo]) * (k - lo)


@dataclass
class Batch:
    bid: int
    requests: list
    key: tuple
    nbytes: int
    handle: object = None    # executor's in-flight token


class Scheduler:
    """Admission by budget and continuous batching, driven by a clock.

    The executor provides: ``request_bytes(req)``, ``batch_bytes(reqs, key)``,
    ``launch(batch) -> token``, ``done(token) -> bool``, ``finish(batch)``,
    ``now() -> float`` (seconds since start) and ``idle()`` (wait a little).
    """

    def __init__(self, executor, budget_bytes: float, max_batch: int = 64,
                 max_in_flight: int = 3, policy: str = "mixed"):
        self.x = executor
        self.budget = float(budget_bytes)
        self.max_batch = max_batch
        self.max_in_flight = max_in_flight
        self.policy = policy
        self.used = 0.0
        self.peak = 0.0
        self.batches = 0

    def reserve(self, r: Request) -> float:
        """Device bytes a request holds from admission to completion."""
        return self.x.request_bytes(r) + self.x.batch_bytes([r], self.key_of(r))

    def key_of(self, r: Request):
        if self.policy == "sequential":
            return ("seq", r.rid)
        refine_pays = getattr(self.x, "refine_pays", None)
        mixed = (self.policy == "mixed" and r.mixed_ok and
                 (refine_pays is None or refine_pays(r.solvedim)))
        return (r.solvedim, "mixed" if mixed else "f64")

    def run(self, trace: list[Request]) -> list[Request]:
        pending = sorted(trace, key=lambda r: r.arrival)
        arrived: list[Request] = []     # queued, not admitted
        admitted: list[Request] = []    # admitted, not launched
        in_flight: list[Batch] = []
        i = 0
        finished = 0
        while finished < len(trace):
            now = self.x.now()
            while i < len(pending) and pending[i].arrival <= now:
                arrived.append(pending[i])
                i += 1
            # completions free memory first
            for b in [b for b in in_flight if self.x.done(b.handle)]:
                t = self.x.now()
                self.x.finish(b)
                for r in b.requests:
                    r.done = t
                self.used -= b.nbytes
                in_flight.remove(b)
                finished += len(b.requests)
            # admission: first come, first served, while a request's iterate
            # and its share of plan scratch fit (a lone request larger than
            # the whole budget still runs, by itself)
            while arrived:
                r = arrived[0]
                need = self.reserve(r)
                if self.used + need > self.budget and (self.used > 0 or admitted):
                    break
                arrived.pop(0)
                r.admitted = now
                self.used += need
                self.peak = max(self.peak, self.used)
                admitted.append(r)
            # launch: the group holding the oldest admitted request
            launched = False
            while admitted and len(in_flight) < self.max_in_flight:
                key = self.key_of(admitted[0])
                group = [r for r in admitted if self.key_of(r) == key][: self.max_batch]
                t_launch = self.x.now()
                for r in group:
                    admitted.remove(r)
                    r.started = t_launch
                    r.batch = self.batches
                b = Batch(self.batches, group, key, sum(self.reserve(r) for r in group))
                self.batches += 1
                b.handle = self.x.launch(b)
                in_flight.append(b)
                launched = True
            if not launched:
                if i < len(pending) and not in_flight and not admitted:
                    self.x.idle(until=pending[i].arrival)
                else:
                    self.x.idle()
        return trace


def report(trace: list[Request]) -> dict:
    lat = [(r.done - r.arrival) * 1e3 for r in trace]
    t0 = min(r.arrival for r in trace)
    t1 = max(r.done for r in trace)
    return {
        "requests": len(trace),
        "solves_per_s": round(len(trace) / (t1 - t0), 1),
        "p50_ms": round(percentile(lat, 0.5), 3),
        "p99_ms": round(percentile(lat, 0.99), 3),
        "mean_ms": round(sum(lat) / len(lat), 3),
        "makespan_s": round(t1 - t0, 4),
    }


# ---------------------------------------------------------------------------
# The CUDA executor
# ---------------------------------------------------------------------------
class ProblemPool:
    """Device-resident FP64 problems (coefficients and a right-hand side)
    with random dominant coefficients as in the 64^3 parity config."""

    def __init__(self, shapes, device="cuda", seed=0):
        import torch

        self.shapes = [tuple(s) for s in shapes]
        self.items = []
        g = torch.Generator(device=device).manual_seed(seed)
        for dims in self.shapes:
            shape = tuple(reversed(dims))

            def u(lo, hi):
                return torch.rand(shape, generator=g, device=device,
                                  dtype=torch.float64) * (hi - lo) + lo

            ds, dl, du, dw = u(-1, 1), u(-1, 1), u(-1, 1), u(-1, 1)
            d = ds.abs() + dl.abs() + du.abs() + dw.abs() + u(1, 2)
            self.items.append({"ds": ds, "dl": dl, "d": d, "du": du, "dw": dw, "b": u(-1, 1)})
        self._free = [[] for _ in self.shapes]   # iterates of finished requests, per problem

    def iterate(self, i):
        """A copy of problem i's right-hand side to solve in place (queued on the
        current stream), in an iterate buffer that a finished request gave back
        when there is one: a server holds its iterate memory instead of asking
        the allocator for every request."""
        x = self._free[i].pop() if self._free[i] else self.items[i]["b"].new_empty(
            self.items[i]["b"].shape)
        x.copy_(self.items[i]["b"])
        return x

    def give_back(self, i, x) -> None:
        """Return an iterate whose request's work has completed on the device."""
        self._free[i].append(x)

    def drop_iterates(self) -> None:
        """Forget the kept iterates (their memory goes back to the allocator)."""
        self._free = [[] for _ in self.shapes]

    def points(self, i) -> int:
        return int(math.prod(self.shapes[i]))

    def nbytes(self) -> int:
        return sum(7 * 8 * self.points(i) for i in range(len(self.shapes)))


class CudaExecutor:
    """Runs batches as plans (or, for the sequential baseline, single calls)."""

    def __init__(self, pool: ProblemPool, refine_steps: int = 1, streams: int = 3,
                 keep_results: bool = False, calibrate: bool = False):
        import torch

        import pentadsolver as ps

        self.ps = ps
        self.torch = torch
        self.pool = pool
        self.refine_steps = refine_steps
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        self.next_stream = 0
        self.keep_results = keep_results
        self.results = {}
        self.status = {}   # request id -> status bits of the batch that solved it
        self.t0 = time.perf_counter()
        self.handle = ps.Handle()
        self._seq_buf = None   # the sequential baseline's one buffer, sized on first use
        # FP64 plans' scratch, one growing buffer per stream: a batch's plan runs
        # after everything queued before it on its stream, so it may reuse it
        self._scratch = [None] * len(self.streams)
        # per solve direction: does the refined form beat plain FP64 here?
        self.calibration = self.measure_costs() if calibrate else None

    def measure_costs(self, reps: int = 3) -> dict:
        """Time a refinement plan against a plain FP64 plan along each solve
        direction on the pool's largest problem (device time, after a warm-up
        execute); the refined form is used only where it was faster."""
        torch, ps = self.torch, self.ps
        big = max(range(len(self.pool.shapes)), key=self.pool.points)
        p = self.pool.items[big]
        out = {}
        for solvedim in range(3):
            g = {"ds": p["ds"], "dl": p["dl"], "d": p["d"], "du": p["du"], "dw": p["dw"],
                 "x": p["b"].clone()}
            ms = {}
            for label, steps in (("fp64", None), ("refined", self.refine_steps)):
                with ps.Plan([g], solvedim, refine_steps=steps, handle=self.handle) as plan:
                    plan.execute()
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    for _ in range(reps):
                        plan.execute()
                    e1.record()
                    torch.cuda.synchronize()
                    ms[label] = e0.elapsed_time(e1) / reps
            out[solvedim] = {"fp64_ms": round(ms["fp64"], 4),
                             "refined_ms": round(ms["refined"], 4),
                             "refine_pays": ms["refined"] < ms["fp64"]}
        return {"problem": list(self.pool.shapes[big]), "per_solvedim": out}

    def refine_pays(self, solvedim: int) -> bool:
        if self.calibration is None:
            return True
        return self.calibration["per_solvedim"][solvedim]["refine_pays"]

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def idle(self, until: float | None = None) -> None:
        if until is not None:
            dt = until - self.now()
            if dt > 2e-4:
                time.sleep(dt - 1e-4)

    def request_bytes(self, r: Request) -> int:
        return 8 * self.pool.points(r.problem)   # its iterate

    def batch_bytes(self, reqs, key) -> int:
        # plan scratch: at most the reference-sized buffer of each grid
        # (refinement: FP32 copies + residual + saved b + an FP32 buffer)
        per = 0
        for r in reqs:
            n = self.pool.points(r.problem)
            mixed = key[1] == "mixed" if key[0] != "seq" else False
            per += n * (20 + 4 + 8 + 36) if mixed else n * 8 * 9
        return per

    def launch(self, b: Batch):
        torch, ps = self.torch, self.ps
        si = self.next_stream
        s = self.streams[si]
        self.next_stream = (self.next_stream + 1) % len(self.streams)
        grids = []
        with torch.cuda.stream(s):
            for r in b.requests:
                p = self.pool.items[r.problem]
                x = self.pool.iterate(r.problem)
                grids.append({"ds": p["ds"], "dl": p["dl"], "d": p["d"], "du": p["du"],
                              "dw": p["dw"], "x": x})
            if b.key[0] == "seq":
                # like the reference's application, one buffer for every call:
                # the reference-sized buffer of the pool's largest need
                r, g = b.requests[0], grids[0]
                if self._seq_buf is None:
                    need = max(ps.buffer_size(list(d), sd, 8) for d in self.pool.shapes
                               for sd in range(3))
                    self._seq_buf = ps.aligned_bytes(need, x.device)
                ps.gpsv_batch(g["ds"], g["dl"], g["d"], g["du"], g["dw"], g["x"], r.solvedim,
                              buffer=self._seq_buf, stream=s, handle=self.handle)
                plan = None
            else:
                steps = self.refine_steps if b.key[1] == "mixed" else None
                scratch = None
                if steps is None:
                    need = ps.plan_sizes(grids, b.key[0], self.handle)[1]
                    if self._scratch[si] is None or self._scratch[si].numel() < need:
                        self._scratch[si] = None
                        self._scratch[si] = ps.aligned_bytes(max(need + need // 4, 256),
                                                             x.device)
                    scratch = self._scratch[si]
                plan = ps.Plan(grids, b.key[0], refine_steps=steps, handle=self.handle,
                               scratch=scratch)
                plan.execute(s)
            ev = torch.cuda.Event()
            ev.record(s)
        if b.key[0] == "seq":
            ev.synchronize()   # the baseline waits for each call
        return (ev, plan, grids, s)

    def done(self, token) -> bool:
        return token[0].query()

    def finish(self, b: Batch) -> None:
        ev, plan, grids, s = b.handle
        # the batch has finished: its status word (the plan's own, or the
        # executor handle's for a single call) says whether any of its
        # kernels met a zero pivot or gave up a wait
        if hasattr(plan, "status_check"):
            bits = plan.status_check(s)[1]
        else:
            bits = self.ps.status_check(s, self.handle)[1]
        for r in b.requests:
            self.status[r.rid] = bits
        if hasattr(plan, "close"):
            plan.close()
        for r, g in zip(b.requests, grids):
            if self.keep_results:
                self.results[r.rid] = g["x"]
            else:
                self.pool.give_back(r.problem, g["x"])
        b.handle = None


def serve(pool: ProblemPool, trace, policy: str, budget_bytes: float, max_batch: int = 64,
          refine_steps: int = 1, keep_results: bool = False, calibrate: bool = False):
    """Run a trace in real time; returns (report, executor, trace).  With
    `calibrate`, the mixed policy first measures where refinement pays."""
    import copy

    tr = copy.deepcopy(trace)
    ex = CudaExecutor(pool, refine_steps=refine_steps, keep_results=keep_results,
                      calibrate=calibrate and policy == "mixed")
    sch = Scheduler(ex, budget_bytes, max_batch=max_batch,
                    max_in_flight=1 if policy == "sequential" else 3, policy=policy)
    ex.torch.cuda.synchronize()
    with no_gc():
        ex.t0 = time.perf_counter()
        sch.run(tr)
        ex.torch.cuda.synchronize()
    rep = report(tr)
    rep.update({"policy": policy, "batches": sch.batches,
                "peak_budget_gb": round(sch.peak / 1e9, 3)})
    if ex.calibration is not None:
        rep["calibration"] = ex.calibration
    return rep, ex, tr


# ---------------------------------------------------------------------------
# The native serving handle (pentadsolver_server_*: admission, batching,
# streams and memory in the library)
# ---------------------------------------------------------------------------
POLICIES = {"fp64": 0, "mixed": 1, "sequential": 2}


class NativeServer:
    """ctypes front end of the library's serving handle; its arena (the HBM
    budget for batch memory) is one device allocation made here."""

    def __init__(self, arena_bytes: int, policy: str = "fp64", streams: int = 3,
                 max_batch: int = 64, max_in_flight: int = 3, refine_steps: int = 1,
                 handle=None, device="cuda"):
        import ctypes

        import torch

        import pentadsolver as ps

        self.ps, self.ct = ps, ctypes
        self.handle = handle
        self.arena = torch.empty(int(arena_bytes) + 256, dtype=torch.uint8, device=device)
        off = (-self.arena.data_ptr()) % 256
        self._arena = self.arena[off:off + int(arena_bytes)]
        self._srv = ctypes.c_void_p(None)
        f = ps._typed("pentadsolver_server_create",
                      [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                       ctypes.POINTER(ctypes.c_void_p)])
        st = f(ps._hval(handle), self._arena.data_ptr(), int(arena_bytes), POLICIES[policy],
               int(streams), int(max_batch), int(max_in_flight), int(refine_steps),
               ctypes.byref(self._srv))
        if st != ps.SUCCESS:
            raise ps.PentadError(st, "server create")
        self._grids = {}   # id -> grid descriptor kept alive until completion
        # the entry points, typed once
        ct = ctypes
        self._submit = ps._typed("pentadsolver_server_submit",
                                 [ct.c_void_p, ct.POINTER(ps.GridDesc), ct.c_int, ct.c_double,
                                  ct.POINTER(ct.c_ulonglong)])
        self._progress = ps._typed("pentadsolver_server_progress", [ct.c_void_p, ct.c_int])
        self._poll = ps._typed("pentadsolver_server_poll",
                               [ct.c_void_p, ct.c_void_p, ct.c_void_p, ct.c_int,
                                ct.POINTER(ct.c_int)])
        self._stats = ps._typed("pentadsolver_server_stats",
                                [ct.c_void_p, ct.c_void_p, ct.c_int])
        self._cap = 1024
        self._ids = (ct.c_ulonglong * self._cap)()
        self._bits = (ct.c_int * self._cap)()

    def submit(self, grid: dict, solvedim: int, tol: float) -> int:
        ct, ps = self.ct, self.ps
        desc = ps._grid_descs([grid])
        rid = ct.c_ulonglong(0)
        st = self._submit(self._srv, desc, int(solvedim), float(tol), ct.byref(rid))
        if st != ps.SUCCESS:
            raise ps.PentadError(st, "server submit")
        self._grids[rid.value] = (desc, grid)
        return int(rid.value)

    def progress(self, wait: bool = False) -> None:
        st = self._progress(self._srv, 1 if wait else 0)
        if st != self.ps.SUCCESS:
            raise self.ps.PentadError(st, "server progress")

    def poll(self) -> list[tuple[int, int]]:
        ct = self.ct
        ids, bits = self._ids, self._bits
        n = ct.c_int(0)
        st = self._poll(self._srv, ids, bits, self._cap, ct.byref(n))
        if st != self.ps.SUCCESS:
            raise self.ps.PentadError(st, "server poll")
        out = [(int(ids[i]), int(bits[i])) for i in range(n.value)]
        for rid, _ in out:
            self._grids.pop(rid, None)
        return out

    def stats(self) -> dict:
        vals = (self.ct.c_size_t * 6)()
        self._stats(self._srv, vals, 6)
        keys = ("queued", "in_flight", "arena_used", "arena_peak", "arena_bytes", "batches")
        return dict(zip(keys, (int(v) for v in vals)))

    def calibrate(self, grid: dict, reps: int = 3) -> dict:
        ct, ps = self.ct, self.ps
        desc = ps._grid_descs([grid])
        ms = (ct.c_double * 6)()
        st = ps._typed("pentadsolver_server_calibrate",
                       [ct.c_void_p, ct.POINTER(ps.GridDesc), ct.c_int, ct.c_void_p])(
            self._srv, desc, int(reps), ms)
        if st != ps.SUCCESS:
            raise ps.PentadError(st, "server calibrate")
        return {d: {"fp64_ms": round(ms[2 * d], 4), "refined_ms": round(ms[2 * d + 1], 4),
                    "refine_pays": ms[2 * d + 1] < ms[2 * d]} for d in range(3)}

    def close(self) -> None:
        if self._srv.value:
            self.ps._typed("pentadsolver_server_destroy", [self.ct.c_void_p])(self._srv)
            self._srv = self.ct.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_native(pool: ProblemPool, trace, policy: str, arena_bytes: float, max_batch: int = 64,
                 refine_steps: int = 1, keep_results: bool = False, calibrate: bool = False,
                 streams: int = 3):
    """Replay a trace in real time through the library's serving handle:
    requests whose arrival time has come are submitted (each with its iterate,
    a copy of the problem's right-hand side) while fewer than three batches'
    worth wait in the handle's queue -- the others wait here, as the Python
    loop's admission holds them, so iterates exist only for requests near the
    device -- the handle batches and launches, and completions are polled.
    Latency counts from arrival.  Returns (report, results, status bits,
    trace)."""
    import copy

    import torch

    tr = copy.deepcopy(trace)
    srv = NativeServer(int(arena_bytes), policy, streams=streams, max_batch=max_batch,
                       refine_steps=refine_steps)
    cal = None
    if calibrate and policy == "mixed":
        big = max(range(len(pool.shapes)), key=pool.points)
        p = pool.items[big]
        cal = srv.calibrate({**{k: p[k] for k in ("ds", "dl", "d", "du", "dw")},
                             "x": p["b"].clone()})
    pending = sorted(tr, key=lambda r: r.arrival)
    by_id, xs, bits = {}, {}, {}
    window = 3 * max_batch
    torch.cuda.synchronize()
    cur = torch.cuda.current_stream()
    gc_ctx = no_gc()
    gc_ctx.__enter__()
    t0 = time.perf_counter()
    i, done = 0, 0
    while done < len(tr):
        now = time.perf_counter() - t0
        submitted = False
        room = window - srv.stats()["queued"]
        while i < len(pending) and pending[i].arrival <= now and room > 0:
            room -= 1
            r = pending[i]
            p = pool.items[r.problem]
            x = pool.iterate(r.problem)
            g = {k: p[k] for k in ("ds", "dl", "d", "du", "dw")}
            g["x"] = x
            rid = srv.submit(g, r.solvedim, r.tol)
            by_id[rid] = r
            xs[rid] = x
            r.admitted = r.started = now
            i += 1
            submitted = True
        if submitted:
            cur.synchronize()   # the iterates' copies, before the server's streams read them
        srv.progress()
        for rid, b in srv.poll():
            r = by_id[rid]
            r.done = time.perf_counter() - t0
            bits[r.rid] = b
            done += 1
            if not keep_results:
                pool.give_back(r.problem, xs.pop(rid))
        if i < len(pending) and srv.stats()["in_flight"] == 0 and not srv.stats()["queued"]:
            dt = pending[i].arrival - (time.perf_counter() - t0)
            if dt > 2e-4:
                time.sleep(dt - 1e-4)
    torch.cuda.synchronize()
    gc_ctx.__exit__(None, None, None)
    rep = report(tr)
    st = srv.stats()
    rep.update({"policy": policy, "native": True, "batches": st["batches"],
                "peak_arena_gb": round(st["arena_peak"] / 1e9, 3)})
    if cal is not None:
        rep["calibration"] = cal
    results = {by_id[rid].rid: x for rid, x in xs.items()} if keep_results else {}
    srv.close()
    return rep, results, bits, tr
