"""The allocation-free entry point pentadsolver_D_gpsv_batch_noalloc.

It exists for callers that cannot call cudaMalloc around a solve (a device
memory pool that owns everything, solve loops where an allocation would
synchronise the device, code that passes no scratch buffer).  It runs the
global-scratch Thomas kernel with its scratch in a fixed 16 MiB device array
inside the library, so its results must agree with the regular entry point
within the parity tolerance (forward error <= 1e-12), call after call, even
though every call reuses the same array.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, solve_dev, to_dev
from oracle import oracle

MAX_BYTES = 16 * 1024 * 1024


def _noalloc():
    fn = ps.lib().pentadsolver_D_gpsv_batch_noalloc
    fn.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _call(dv, solvedim, stream=None):
    x = dv["x"]
    dims = ps.dims_of(x)
    sp = None if stream is None else stream.cuda_stream
    return _noalloc()(None, *(int(dv[k].data_ptr()) for k in NAMES), ps._dims(dims), len(dims),
                      int(solvedim), sp)


def test_noalloc_rejects_grids_beyond_its_array():
    # 128^3 needs 3 * 128^3 * 8 = 48 MiB of scratch: refused before any device work
    dims = [128, 128, 128]
    st = _noalloc()(None, 1, 1, 1, 1, 1, 1, ps._dims(dims), 3, 0, None)
    assert st == ps.INVALID_VALUE
    # and the usual shape rules hold
    st = _noalloc()(None, 1, 1, 1, 1, 1, 1, ps._dims([4, 8, 8]), 3, 0, None)
    assert st == ps.INVALID_VALUE
    # the largest grid that fits is accepted by the size check (88^3 < 699,050 points)
    assert 3 * 88 ** 3 * 8 <= MAX_BYTES < 3 * 89 ** 3 * 8


@pytest.mark.parametrize("dims, solvedim", [([699051, 1, 1], 0), ([699051], 0),
                                            ([1, 699051, 1], 1), ([3, 233017, 1], 1)])
def test_noalloc_rejects_one_point_past_its_array(dims, solvedim):
    # 699,051 points need 3 * 699,051 * 8 = 16,777,224 bytes: 8 past the array.
    # Rejected by the size check itself, before any device work (pointers are
    # placeholders that nothing dereferences).
    assert 3 * 8 * int(np.prod(dims)) == MAX_BYTES + 8
    st = _noalloc()(None, 1, 1, 1, 1, 1, 1, ps._dims(dims), len(dims), solvedim, None)
    assert st == ps.INVALID_VALUE


def test_noalloc_shape_rules_match_the_regular_entry_point():
    # dimensions whose product overflows 64 bits, a line longer than 2^24 rows,
    # and a non-positive extent are refused exactly as pentadsolver_buffer_size_ex
    # refuses them, without touching the device
    for dims, solvedim in (([1 << 30] * 8, 0), ([(1 << 24) + 1, 1, 1], 0), ([16, 0, 16], 0),
                           ([16, 16, 16], 3), ([16] * 9, 0)):
        st = _noalloc()(None, 1, 1, 1, 1, 1, 1, ps._dims(dims), len(dims), solvedim, None)
        assert st == ps.INVALID_VALUE, dims
        with pytest.raises(ps.PentadError):
            ps.buffer_size(dims, solvedim)


def test_noalloc_accepts_the_largest_grid_without_a_device():
    # 699,050 points pass the size check; with no CUDA device the call then
    # stops at binding the handle (nothing is launched)
    import torch

    if torch.cuda.is_available():
        pytest.skip("only meaningful where no device can be bound")
    st = _noalloc()(None, 1, 1, 1, 1, 1, 1, ps._dims([699050, 1, 1]), 3, 0, None)
    assert st == ps.NOT_INITIALIZED


@pytest.mark.gpu
def test_noalloc_matches_regular_entry_point_on_consecutive_calls(cuda):
    import torch

    cases = [((40, 24, 18), 1, 101), ((33, 17, 29), 2, 202), ((88, 88, 88), 0, 303)]
    stream = torch.cuda.Stream()
    expected, got = [], []
    for dims, axis, seed in cases:
        co = fixtures.random_dominant(dims, seed, np.float64)
        ref = to_dev(co)
        solve_dev(ref, axis)          # the regular entry point (caller buffer)
        expected.append(ref["x"])
        dv = to_dev(co)
        got.append(dv)
    torch.cuda.synchronize()
    # the three allocation-free calls back to back on one stream, no sync between
    for (dims, axis, _), dv in zip(cases, got):
        assert _call(dv, axis, stream) == ps.SUCCESS
    stream.synchronize()
    for (dims, axis, seed), dv, exp in zip(cases, got, expected):
        e = fwd_err(dv["x"].cpu().numpy(), exp.cpu().numpy())
        assert e <= 1e-12, (dims, axis, e)
    # and against the oracle for the first case
    dims, axis, seed = cases[0]
    co = fixtures.random_dominant(dims, seed, np.float64)
    oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], co["x"], axis)
    assert fwd_err(got[0]["x"].cpu().numpy(), co["x"]) <= 1e-12
    st, bits = ps.status_check()
    assert st == ps.SUCCESS and bits == 0


@pytest.mark.gpu
def test_noalloc_repeated_calls_on_the_same_grid(cuda):
    dims = (64, 48, 40)
    co = fixtures.random_dominant(dims, 7, np.float64)
    ref = co["x"].copy()
    dv = to_dev(co)
    for axis in (0, 1, 2, 0):
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
        assert _call(dv, axis) == ps.SUCCESS
    import torch

    torch.cuda.synchronize()
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12
