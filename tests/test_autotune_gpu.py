"""The autotuner on the GPU: it times the applicable candidates, the choice
it applies to a handle is the variant that then runs, results stay correct,
and it picks a plan's CTA count."""
import numpy as np
import pytest

import autotune
import fixtures
import pentadsolver as ps
from gpu_util import NAMES, direction, fwd_err, solve_dev, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solvedim", [0, 1])
def test_tune_and_apply(cuda, solvedim, tmp_path):
    import torch

    dims = (64, 48, 40)
    t = autotune.Autotuner(cache_path=tmp_path / "t.json", reps=2)
    res = t.tune_solve(dims, solvedim, torch.float64)
    labels = [r["label"] for r in res["table"]]
    assert len(labels) >= 3 and res["best"] in res["table"]
    co = fixtures.random_dominant(dims, 21, np.float64)
    ref = co["x"].copy()
    oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, solvedim)
    dv = to_dev(co)
    with ps.Handle() as h:
        best = t.apply(h, dims, solvedim, torch.float64)
        solve_dev(dv, solvedim, handle=h)
        assert h.variant_that_ran(direction(3, solvedim)) == best["variant"]
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12


def test_tune_plan_ctas(cuda):
    dims_list = [(40, 24, 18), (33, 17, 29), (64, 20, 12)]
    grids = [to_dev(fixtures.random_dominant(d, 5 + i, np.float64)) for i, d in enumerate(dims_list)]
    res = autotune.Autotuner(reps=2).tune_plan(grids, 1)
    assert res["best"]["ctas"] >= 1 and len(res["table"]) == len(autotune.CTA_CANDIDATES)
