"""GPU: solves issued back to back on one stream, with programmatic dependent
launches between the TMEM kernels, give the bits of the same solves each
followed by a device synchronisation.

The TMEM general kernel and the shared-factorisation kernel let the next solve
on the stream start its on-chip prologue before they finish; each touches
global memory only after ``griddepcontrol.wait``.  A chain that mixes the two
families on one buffer (the general kernel's scratch and the factor-table cache
share it) and reads each solve's result in the next one would expose any
access issued before that wait.
"""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

# x general, y shared factorisation, z general; and shared factorisation only
CHAINS = [("thomas-pcr", "shared-fact", "thomas-pcr"), ("shared-fact",) * 3,
          ("thomas-pcr",) * 3]


def run_chain(dv, algos, iterations, sync_each: bool, buf):
    import torch

    with ps.Handle() as h:
        for a, algo in enumerate(algos):
            h.set_algo(a, algo)
        for _ in range(iterations):
            for axis in range(3):
                ps.gpsv_batch(*(dv[k] for k in NAMES), axis, buffer=buf, handle=h)
                if sync_each:
                    torch.cuda.synchronize()
        torch.cuda.synchronize()
        ran = [h.kernel_that_ran(a) for a in range(3)]
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
    return dv["x"].clone(), ran


@pytest.mark.parametrize("algos", CHAINS)
@pytest.mark.parametrize("dims", [(64, 48, 40), (128, 96, 80)])
def test_back_to_back_equals_synchronised(cuda, algos, dims):
    import torch

    co = fixtures.adi_constant(dims)
    buf = ps.alloc_buffer(list(dims), 0, torch.float64, cuda)
    want, ran = run_chain(to_dev(co), algos, 4, True, buf)
    assert ran == list(algos), ran
    for _ in range(2):
        got, _ = run_chain(to_dev(co), algos, 4, False, buf)
        assert torch.equal(got.view(torch.int64), want.view(torch.int64))
    assert ps.status_check()[1] == 0
    ref = co["x"].astype(np.float64)
    for _ in range(4):
        for axis in range(3):
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
    assert fwd_err(want.cpu().numpy(), ref) <= 1e-12
