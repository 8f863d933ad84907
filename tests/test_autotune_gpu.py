"""The library's autotuner on the GPU.

* It times the applicable candidates on a problem, and the fastest becomes
  the automatic choice of every handle for that shape class -- a handle with
  no choice of its own then runs exactly the tuned variant, with results
  that still equal the oracle's.
* A C++ caller of the reference's interface picks tuned choices up with no
  code change: the reference's ADI app (``apps/adi_cuda.cu``, unchanged,
  built on this library) reads the table from PENTA_TUNING_CACHE and runs the
  kernel family the table names.
* Plans take their CTA count from the table.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

import autotune
import fixtures
import pentadsolver as ps
from gpu_util import NAMES, direction, fwd_err, solve_dev, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


@pytest.fixture(autouse=True)
def _empty_table():
    ps.tuning_clear()
    yield
    ps.tuning_clear()


@pytest.mark.parametrize("solvedim", [0, 1])
def test_tuned_choice_becomes_the_automatic_one(cuda, solvedim, tmp_path):
    import torch

    dims = (64, 48, 40)
    t = autotune.Autotuner(cache_path=tmp_path / "t.tsv", reps=2)
    res = t.tune_solve(dims, solvedim, torch.float64)
    table = res["table"]
    assert len(table) >= 3 and res["best"] == table[0]
    assert table[0]["ms"] == min(r["ms"] for r in table)
    assert len({r["variant"] for r in table}) == len(table)
    assert (tmp_path / "t.tsv").exists()
    co = fixtures.random_dominant(dims, 21, np.float64)
    ref = co["x"].copy()
    oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, solvedim)
    dv = to_dev(co)
    d = direction(3, solvedim)
    with ps.Handle() as h:   # no choice of its own: the table decides
        solve_dev(dv, solvedim, handle=h)
        assert h.variant_that_ran(d) == table[0]["variant"]
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12
    # the slowest candidate, forced into the table, is what runs next
    slow = table[-1]
    key = t.key(dims, solvedim, torch.float64)
    ps.tuning_set(key, slow["spec"], slow["algo"], slow["lanes"], 0, slow["ms"])
    dv = to_dev(co)
    with ps.Handle() as h:
        solve_dev(dv, solvedim, handle=h)
        assert h.variant_that_ran(d) == slow["variant"]
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12


def test_autotune_keeps_the_right_hand_side_when_asked(cuda):
    import torch

    co = fixtures.random_dominant((40, 24, 18), 3, np.float64)
    dv = to_dev(co)
    b = dv["x"].clone()
    save = torch.empty_like(b)
    rows = ps.autotune_solve(*(dv[k] for k in NAMES), 2, reps=1, x_save=save)
    assert rows and torch.equal(dv["x"], b)


def test_a_reference_caller_follows_the_tuning_file(cuda, tmp_path):
    exe = REF / "app_cuda_b200"
    if not exe.exists():
        pytest.skip(f"{exe} not built (oracle/Makefile ref)")
    import torch

    gpu = torch.cuda.get_device_name()
    path = tmp_path / "tune.tsv"
    # the app's 64^3 FP64 x solve sent to the global-scratch kernel by the table
    key = ps.tuning_key([64, 64, 64], 0, 8, "solve", gpu)
    path.write_text(f"{key}\tauto\tnaive\t0\t0\t1\n")
    env = {k: v for k, v in os.environ.items() if not k.startswith("PENTA_")}
    runs = {}
    for label, extra in (("plain", {}), ("tuned", {"PENTA_TUNING_CACHE": str(path)})):
        r = subprocess.run([str(exe), "64", "5", "double"], env={**env, **extra},
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        f = [ln for ln in r.stdout.splitlines() if ln.startswith("CSV,")][-1].split(",")
        runs[label] = (f[2], f[4], f[6])
    assert runs["plain"] == ("thomas-pcr",) * 3
    assert runs["tuned"] == ("naive", "thomas-pcr", "thomas-pcr")


def test_plans_take_their_cta_count_from_the_table(cuda):
    import torch

    dims_list = [(40, 24, 18), (33, 17, 29), (64, 20, 12)]
    grids = [to_dev(fixtures.random_dominant(d, 5 + i, np.float64))
             for i, d in enumerate(dims_list)]
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    res = autotune.Autotuner(reps=2).tune_plan(grids, 1)
    best = res["best"]["ctas"]
    assert best in {max(1, int(sms * f)) for f in autotune.CTA_FRACTIONS}
    with ps.Plan(grids, 1) as plan:      # ctas = 0: the table's count
        assert f"ctas={best}" in plan.describe()
    ps.tuning_clear()
    with ps.Plan(grids, 1) as plan:
        assert f"ctas={sms}" in plan.describe()
    # results are those of the oracle whatever the CTA count
    refs = []
    for i, d in enumerate(dims_list):
        co = fixtures.random_dominant(d, 5 + i, np.float64)
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], co["x"], 1)
        refs.append(co["x"])
    fresh = [to_dev(fixtures.random_dominant(d, 5 + i, np.float64))
             for i, d in enumerate(dims_list)]
    with ps.Plan(fresh, 1, ctas=max(1, sms // 2)) as plan:
        plan.execute()
        assert plan.status_check() == (ps.SUCCESS, 0)
    for g, r in zip(fresh, refs):
        assert fwd_err(g["x"].cpu().numpy(), r) <= 1e-12
