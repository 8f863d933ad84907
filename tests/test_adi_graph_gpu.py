"""GPU: ADI steps captured into one CUDA graph (adi.AdiGraph) give the same
bits as the same calls made one by one, for the general kernels and for
shared factorisation (whose tables stay cached in the buffer across steps),
and agree with the oracle (forward error <= 1e-12 after each run)."""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from adi import AdiGraph
from gpu_util import NAMES, fwd_err, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu


def eager(dv, iterations, algo=None):
    import torch

    buf = ps.alloc_buffer(ps.dims_of(dv["x"]), 0, dv["x"].dtype)
    with ps.Handle() as h:
        if algo is not None:
            for a in range(3):
                h.set_algo(a, algo)
        for _ in range(iterations):
            for axis in range(3):
                ps.gpsv_batch(*(dv[k] for k in NAMES), axis, buffer=buf, handle=h)
        torch.cuda.synchronize()
    return dv["x"].clone()


@pytest.mark.parametrize("algo,dims", [(None, (48, 40, 36)), ("shared-fact", (64, 48, 40))])
def test_adi_graph_matches_calls_and_oracle(cuda, algo, dims):
    import torch

    co = fixtures.random_dominant(dims, 77, np.float64) if algo is None \
        else fixtures.adi_constant(dims)
    iterations = 3
    want = eager(to_dev(co), iterations, algo)
    dv = to_dev(co)
    with AdiGraph(*(dv[k] for k in NAMES), iterations=iterations, algo=algo) as g:
        # capture left x alone
        assert torch.equal(dv["x"], to_dev(co)["x"])
        assert g.launches == 3 * iterations
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(dv["x"], want)
        fam = g.kernels()
        # a second replay continues from the first one's result
        g.replay()
        torch.cuda.synchronize()
        twice = dv["x"].clone()
        assert ps.status_check(handle=g.handle) == (ps.SUCCESS, 0)   # the graph's handle
    if algo is not None:
        assert fam == [algo] * 3, fam
    ref = co["x"].astype(np.float64)
    for _ in range(2 * iterations):
        for axis in range(3):
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
    assert fwd_err(twice.cpu().numpy(), ref) <= 1e-12
