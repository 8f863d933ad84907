"""Status words on the GPU: per-handle and per-plan attribution, read-and-clear
by one atomic exchange, and the bounded waits.

The reference reports nothing from its kernels (``launch_succeeded`` only
checks the launch, ``src/cuda/singlenode/pentad_cuda.cu:26-37``).  Here every
kernel ORs status bits into the word of the handle or plan that launched it:
bit 0 a zero or non-finite pivot, bit 1 a wait inside the kernel that ran out.

The timeout case makes a wait run out on purpose, the way the failure tests of
this project are allowed to: a kernel waits on an mbarrier that only one of its
two expected arrivals ever reaches, gives up after one millisecond and raises
bit 1.  Nothing faults or hangs; the same context solves correctly afterwards.
"""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, solve_dev, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu


def _zero_pivot_problem(dims=(16, 8, 8), seed=3):
    co = fixtures.random_dominant(dims, seed, np.float64)
    co["d"][2, 3, 0] = 0.0      # first row of one x line: pivot exactly zero
    co["dl"][2, 3, 1] = 0.0
    co["ds"][2, 3, 2] = 0.0
    return co


def test_bounded_wait_runs_out_and_is_reported(cuda):
    import torch

    with ps.Handle() as h:
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
        stream = torch.cuda.Stream()
        assert ps.selftest_bounded_wait(1000, stream=stream, handle=h) == ps.SUCCESS
        st, bits = ps.status_check(stream=stream, handle=h)
        assert bits == ps.TIMEOUT_BIT and st == ps.SUCCESS
        # read and cleared in one exchange: nothing left for the next check
        assert ps.status_check(stream=stream, handle=h) == (ps.SUCCESS, 0)
        # the NULL handle's word never saw it
        assert ps.status_check()[1] == 0
        # the context is still usable: a solve on the same handle is exact
        co = fixtures.random_dominant((24, 20, 12), 77, np.float64)
        dv = to_dev(co)
        solve_dev(dv, 1, handle=h, check_status=False)
        torch.cuda.synchronize()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], co["x"], 1)
        assert fwd_err(dv["x"].cpu().numpy(), co["x"]) <= 1e-12
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
    assert ps.selftest_bounded_wait(0) == ps.INVALID_VALUE


def test_status_words_are_per_handle(cuda):
    import torch

    bad, good = ps.Handle(), ps.Handle()
    try:
        dv_bad = to_dev(_zero_pivot_problem())
        dv_good = to_dev(fixtures.random_dominant((16, 8, 8), 4, np.float64))
        s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
        solve_dev(dv_bad, 0, handle=bad, stream=s1, check_status=False)
        solve_dev(dv_good, 0, handle=good, stream=s2, check_status=False)
        torch.cuda.synchronize()
        assert ps.status_check(stream=s2, handle=good) == (ps.SUCCESS, 0)
        assert ps.status_check()[1] == 0
        st, bits = ps.status_check(stream=s1, handle=bad)
        assert st == ps.ZERO_PIVOT and bits & ps.ZERO_PIVOT_BIT
        assert ps.status_check(stream=s1, handle=bad) == (ps.SUCCESS, 0)
    finally:
        bad.close()
        good.close()
    # a new handle (which may reuse a released slot) starts clean
    with ps.Handle() as h:
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)


@pytest.mark.parametrize("solvedim", [0, 2])
def test_status_words_are_per_plan(cuda, solvedim):
    probs = [_zero_pivot_problem(), fixtures.random_dominant((20, 12, 9), 5, np.float64)]
    if solvedim == 2:   # put the zero pivot on a z line instead
        probs[0] = fixtures.random_dominant((16, 8, 8), 3, np.float64)
        probs[0]["d"][0, 3, 2] = 0.0
        probs[0]["dl"][1, 3, 2] = 0.0
        probs[0]["ds"][2, 3, 2] = 0.0
    clean = [fixtures.random_dominant((18, 10, 7), 6, np.float64)]
    with ps.Plan([to_dev(co) for co in probs], solvedim) as p_bad, \
            ps.Plan([to_dev(co) for co in clean], solvedim) as p_good:
        p_bad.execute()
        p_good.execute()
        assert p_good.status_check() == (ps.SUCCESS, 0)
        assert ps.status_check()[1] == 0
        st, bits = p_bad.status_check()
        assert st == ps.ZERO_PIVOT and bits & ps.ZERO_PIVOT_BIT
        assert p_bad.status_check() == (ps.SUCCESS, 0)
