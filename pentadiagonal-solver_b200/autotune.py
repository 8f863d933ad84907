"""Autotuner for the solver's kernel choices.

For one solve shape (precision, direction, line length n, number of lines) it
times every applicable candidate on a synthetic diagonally dominant problem
of that shape and keeps the fastest:

  * the Tensor-Memory kernel's variants (forward ring and read-back stages),
  * the older TMA kernels (automatic variant),
  * the cp.async kernel with two partitions (two lanes) or one lane per line
    (the reference's PENTA_PCR_LANES knob).

For a plan (many grids, one launch) it picks the number of CTAs.  Results are
kept per (GPU, precision, direction class, n bucket, lines bucket) in memory
and, when a path is given, in a JSON file, so a serving process tunes once.
Candidates are applied per handle and direction with
``pentadsolver_set_tuning`` and ``pentadsolver_set_algo``.
"""
from __future__ import annotations

import json
import math
import os
from pathlib import Path

import pentadsolver as ps

# (label, tuning spec, algorithm, pcr lanes)
SOLVE_CANDIDATES = [
    ("tmem 2/4", "tmem=2,4", "thomas-pcr", 2),
    ("tmem 2/3", "tmem=2,3", "thomas-pcr", 2),
    ("tmem 3/4", "tmem=3,4", "thomas-pcr", 2),
    ("tmem 3/3", "tmem=3,3", "thomas-pcr", 2),
    ("tmem 3/2", "tmem=3,2", "thomas-pcr", 2),
    ("tmem 4/3", "tmem=4,3", "thomas-pcr", 2),
    ("tma", "no-tmem", "thomas-pcr", 2),
    ("cp.async P2", "no-tma", "thomas-pcr", 2),
    ("cp.async P1", "no-tma", "thomas-pcr", 1),
]
CTA_CANDIDATES = (1.0, 0.9, 0.75, 0.5)


def _bucket(v: int) -> int:
    return 1 << max(0, math.ceil(math.log2(max(1, v))))


def problem(dims, dtype, device="cuda", seed=0):
    """Synthetic random dominant problem (config-0 distribution) on the device."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    shape = tuple(reversed(list(dims)))

    def u(lo, hi):
        return torch.rand(shape, generator=g, device=device, dtype=torch.float64) * (hi - lo) + lo

    ds, dl, du, dw = u(-1, 1), u(-1, 1), u(-1, 1), u(-1, 1)
    d = ds.abs() + dl.abs() + du.abs() + dw.abs() + u(1, 2)
    out = {"ds": ds, "dl": dl, "d": d, "du": du, "dw": dw, "x": u(-1, 1)}
    return {k: v.to(dtype) for k, v in out.items()}


class Autotuner:
    def __init__(self, cache_path: str | os.PathLike | None = None, reps: int = 5,
                 time_fn=None):
        self.cache_path = Path(cache_path) if cache_path else None
        self.reps = reps
        self.cache: dict[str, dict] = {}
        self._time_fn = time_fn or self._time_cuda
        if self.cache_path and self.cache_path.exists():
            self.cache = json.loads(self.cache_path.read_text())

    # -- keys and persistence --------------------------------------------------
    @staticmethod
    def gpu_name() -> str:
        try:
            import torch

            return torch.cuda.get_device_name()
        except Exception:
            return "unknown"

    def key(self, dims, solvedim, dtype, kind="solve") -> str:
        import torch

        n = int(dims[solvedim])
        lines = int(math.prod(dims)) // n
        prec = "f64" if dtype == torch.float64 else "f32"
        cls = "x" if solvedim == 0 else "yz"
        return f"{self.gpu_name()}|{kind}|{prec}|{cls}|n{_bucket(n)}|l{_bucket(lines)}"

    def save(self) -> None:
        if self.cache_path:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            self.cache_path.write_text(json.dumps(self.cache, indent=1, sort_keys=True))

    # -- timing ------------------------------------------------------------------
    def _time_cuda(self, fn) -> float:
        import torch

        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(self.reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / self.reps

    # -- single solves -----------------------------------------------------------
    def tune_solve(self, dims, solvedim, dtype) -> dict:
        """Time the candidates on this shape; returns the best one and the table."""
        k = self.key(dims, solvedim, dtype)
        if k in self.cache:
            return self.cache[k]
        p = problem(dims, dtype)
        buf = ps.alloc_buffer(list(dims), solvedim, dtype, p["x"].device)
        d = ps.DIR_X if solvedim == 0 else (ps.DIR_OUTERMOST if solvedim == len(dims) - 1
                                            else ps.DIR_MIDDLE)
        table, seen = [], set()
        with ps.Handle() as h:
            for label, spec, algo, lanes in SOLVE_CANDIDATES:
                ps.set_tuning(h, d, spec)
                h.set_algo(d, algo, lanes)
                x0 = p["x"].clone()

                def run():
                    ps.gpsv_batch(p["ds"], p["dl"], p["d"], p["du"], p["dw"], x0, solvedim,
                                  buffer=buf, handle=h)

                run()
                variant = h.variant_that_ran(d)
                if variant in seen:      # the shape sent this candidate elsewhere
                    continue
                seen.add(variant)
                ms = self._time_fn(run)
                table.append({"label": label, "spec": spec, "algo": algo, "lanes": lanes,
                              "variant": variant, "ms": ms})
        best = min(table, key=lambda r: r["ms"])
        out = {"best": best, "table": table}
        self.cache[k] = out
        self.save()
        return out

    def apply(self, handle, dims, solvedim, dtype) -> dict:
        """Tune (or look up) and set the handle's choice for this direction."""
        r = self.tune_solve(dims, solvedim, dtype)["best"]
        d = ps.DIR_X if solvedim == 0 else (ps.DIR_OUTERMOST if solvedim == len(dims) - 1
                                            else ps.DIR_MIDDLE)
        ps.set_tuning(handle, d, r["spec"])
        handle.set_algo(d, r["algo"], r["lanes"])
        return r

    # -- plans ---------------------------------------------------------------------
    def tune_plan(self, grids, solvedim, refine_steps=None) -> dict:
        """Pick the CTA count of a plan over these grids (dicts of tensors;
        their x is restored after each timing)."""
        import torch

        sms = torch.cuda.get_device_properties(grids[0]["x"].device).multi_processor_count
        saved = [g["x"].clone() for g in grids]
        table = []
        for f in CTA_CANDIDATES:
            ctas = max(1, int(sms * f))
            with ps.Plan(grids, solvedim, refine_steps=refine_steps, ctas=ctas) as plan:
                ms = self._time_fn(plan.execute)
            table.append({"ctas": ctas, "ms": ms})
        for g, s in zip(grids, saved):
            g["x"].copy_(s)
        best = min(table, key=lambda r: r["ms"])
        return {"best": best, "table": table}
