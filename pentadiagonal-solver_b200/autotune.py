"""Autotuner front end: the library's own tuner and tuning table from Python.

The tuning itself lives in the C ABI (``pentadsolver_autotune_solve``,
``pentadsolver_autotune_plan``): for one solve shape it times every applicable
kernel choice on the device -- the Tensor-Memory kernel's ring variants, the
older TMA kernels, the cp.async kernel with two lanes or one lane per line
(the reference's PENTA_PCR_LANES knob) -- and for a plan the number of CTAs,
and records the fastest in a process-wide table keyed by shape class
(GPU, solve or plan, precision, x or y/z, line length and number of lines
rounded up to powers of two).  Every handle's automatic selection and plan
creation consult that table, and the library reads it at first use from the
file named by PENTA_TUNING_CACHE -- so a C++ caller of the reference's
interface gets tuned kernels by setting one environment variable.

This module adds what a Python process wants around it: synthetic problems
of a shape, a cache file that is loaded on start and saved after each tuning,
and explicit per-handle application.
"""
from __future__ import annotations

import math
import os
from pathlib import Path

import pentadsolver as ps

CTA_FRACTIONS = (1.0, 0.9, 0.75, 0.5)  # pentadsolver_autotune_plan's candidates


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


def _direction(dims, solvedim) -> int:
    return ps.DIR_X if solvedim == 0 else (ps.DIR_OUTERMOST if solvedim == len(dims) - 1
                                           else ps.DIR_MIDDLE)


class Autotuner:
    """Tunes through the library and keeps its table in ``cache_path``."""

    def __init__(self, cache_path: str | os.PathLike | None = None, reps: int = 5):
        self.cache_path = Path(cache_path) if cache_path else None
        self.reps = reps
        if self.cache_path and self.cache_path.exists():
            ps.tuning_load(self.cache_path)

    @staticmethod
    def gpu_name() -> str:
        try:
            import torch

            return torch.cuda.get_device_name()
        except Exception:
            return "unknown"

    def key(self, dims, solvedim, dtype, kind="solve", gpu_name=None) -> str:
        import torch

        eb = 8 if dtype == torch.float64 else 4
        return ps.tuning_key(list(dims), solvedim, eb, kind,
                             gpu_name if gpu_name is not None else self.gpu_name())

    def save(self) -> None:
        if self.cache_path:
            self.cache_path.parent.mkdir(parents=True, exist_ok=True)
            ps.tuning_save(self.cache_path)

    # -- single solves -----------------------------------------------------------
    def tune_solve(self, dims, solvedim, dtype) -> dict:
        """The table's choice for this shape class, timing the candidates on a
        synthetic problem of this shape first when the table has none:
        {"best": entry, "table": rows timed now (empty when cached)}."""
        k = self.key(dims, solvedim, dtype)
        hit = ps.tuning_lookup(k)
        if hit is not None:
            return {"best": hit, "table": []}
        p = problem(dims, dtype)
        rows = ps.autotune_solve(p["ds"], p["dl"], p["d"], p["du"], p["dw"], p["x"], solvedim,
                                 reps=self.reps)
        self.save()
        return {"best": rows[0], "table": rows}

    def apply(self, handle, dims, solvedim, dtype) -> dict:
        """Tune (or look up) and fix the choice on `handle` for this direction
        (explicitly; handles without a choice of their own use the table)."""
        r = self.tune_solve(dims, solvedim, dtype)["best"]
        d = _direction(dims, solvedim)
        ps.set_tuning(handle, d, r["spec"])
        handle.set_algo(d, r["algo"], r["lanes"])
        return r

    # -- plans ---------------------------------------------------------------------
    def tune_plan(self, grids, solvedim, refine_steps=None) -> dict:
        """The CTA count of a plan over these grids (dicts of tensors; their x
        is restored afterwards), recorded for plans of this class."""
        saved = [g["x"].clone() for g in grids]
        with ps.Plan(grids, solvedim, refine_steps=refine_steps) as plan:
            ctas = plan.autotune(self.reps)
        for g, s in zip(grids, saved):
            g["x"].copy_(s)
        self.save()
        return {"best": {"ctas": ctas}}


def main(argv=None) -> None:
    """Tune from the command line: every candidate's time for each solve
    direction of one grid, fastest first, recorded in the cache file."""
    import argparse

    import torch

    ap = argparse.ArgumentParser(description=main.__doc__.split("\n")[0])
    ap.add_argument("--dims", type=int, nargs="+", required=True, help="t_dims, x first")
    ap.add_argument("--solvedims", type=int, nargs="+", default=None)
    ap.add_argument("--dtype", choices=("f64", "f32"), default="f64")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--cache", default=None, help="tuning table file to load and save")
    args = ap.parse_args(argv)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    tuner = Autotuner(cache_path=args.cache, reps=args.reps)
    ps.tuning_clear()
    p = problem(args.dims, dtype)
    for sd in args.solvedims if args.solvedims is not None else range(len(args.dims)):
        rows = ps.autotune_solve(p["ds"], p["dl"], p["d"], p["du"], p["dw"], p["x"], sd,
                                 reps=args.reps)
        print(f"dims {args.dims} {args.dtype} solvedim {sd}:")
        for r in rows:
            print(f"  {r['ms'] * 1e3:9.1f} us  {r['label']:12s} {r['variant']}")
    tuner.save()


if __name__ == "__main__":
    main()

