"""GPU parity of the shared-factorisation kernels (PENTA_*ALGO=shared-fact).

Shared factorisation solves every line with line 0's coefficients
(src/cuda/singlenode/pentad_cuda.cu:957-1127), so the inputs here give every
line of the solve direction the same coefficient profile (random along the
line, identical across lines) and the oracle solves the same arrays with the
general algorithm.  Tolerances as for the general kernels: forward error
<= 1e-12 (FP64) and <= 1e-5 (FP32).
"""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, direction, fwd_err, solve_dev, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

FWD_TOL = {np.float64: 1e-12, np.float32: 1e-5}


def shared_problem(dims, solvedim, seed, dtype):
    """Random dominant coefficients of one line, repeated on every line along
    ``solvedim``; an independent random right-hand side per point."""
    co = fixtures.random_dominant(dims, seed, dtype)
    ax = len(dims) - 1 - solvedim
    for k in NAMES[:-1]:
        idx = [0] * co[k].ndim
        idx[ax] = slice(None)
        prof = co[k][tuple(idx)]                     # line 0's profile
        shape = [1] * co[k].ndim
        shape[ax] = -1
        co[k] = np.ascontiguousarray(np.broadcast_to(prof.reshape(shape), co[k].shape))
    return co


def oracle_solution(co, solvedim):
    ref = {k: co[k].astype(np.float64) for k in NAMES}
    oracle.solve(ref["ds"], ref["dl"], ref["d"], ref["du"], ref["dw"], ref["x"], solvedim)
    return ref["x"]


def shared_solve(co, solvedim, dims, buffer="default", check_status=True, status=None):
    """Shared-factorisation solve on a handle of its own; with `status` (a
    list), the handle's (status, bits) are appended to it."""
    dv = to_dev(co)
    dirn = direction(len(dims), solvedim)
    with ps.Handle() as h:
        h.set_algo(dirn, "shared-fact")
        if buffer is None:
            ps.gpsv_batch(*(dv[k] for k in NAMES), solvedim, buffer=None, handle=h)
            assert ps.status_check(handle=h)[1] == 0
        elif isinstance(buffer, str):
            solve_dev(dv, solvedim, handle=h, check_status=check_status)
        else:
            solve_dev(dv, solvedim, handle=h, buffer=buffer, check_status=check_status)
        fam, var = h.kernel_that_ran(dirn), h.variant_that_ran(dirn)
        if status is not None:
            status.append(ps.status_check(handle=h))
    assert fam == "shared-fact", fam
    return dv["x"].cpu().numpy(), var


SHAPES = [(64, 64, 64), (48, 20, 33), (40, 24, 18), (256, 3, 5), (6, 40, 21), (33, 17, 6),
          (300, 5, 4), (5, 6, 300), (20, 36, 9), (512, 6, 5), (18, 32, 20)]


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_shared_fact_matches_oracle_every_direction(cuda, dims, dtype):
    eb = np.dtype(dtype).itemsize
    for solvedim in range(3):
        if dims[solvedim] <= 4:
            continue
        co = shared_problem(dims, solvedim, 900 + solvedim, dtype)
        ref = oracle_solution(co, solvedim)
        got, var = shared_solve(co, solvedim, dims)
        assert fwd_err(got, ref) <= FWD_TOL[dtype], (dims, solvedim, var)
        # the Tensor-Memory kernel takes aligned lines split into two halves of
        # m = R ceil(n / 2R) rows, m <= 256 (FP64) / 512 (FP32), with two real
        # rows in the lower half; everything else uses the per-line kernel
        n = dims[solvedim]
        inner = int(np.prod(dims[:solvedim]))
        r = 128 // eb  # rows per stage
        m = r * -(-n // (2 * r))
        aligned = (n * eb) % 16 == 0 if solvedim == 0 else (inner > 1 and (inner * eb) % 16 == 0)
        tm = aligned and m <= (256 if eb == 8 else 512) and n - m >= 2
        assert ("tmem" in var) == tm, (dims, solvedim, var)


def test_shared_fact_table_cache_follows_the_coefficients(cuda):
    """Repeated calls with one buffer reuse the cached table (same bits);
    new coefficients, or a general solve that reused the buffer in between,
    must not leave a stale table behind."""
    import torch

    dims = (64, 48, 40)
    for solvedim in (0, 1, 2):
        buf = ps.alloc_buffer(list(dims), 0, torch.float64)
        a = shared_problem(dims, solvedim, 11, np.float64)
        b = shared_problem(dims, solvedim, 12, np.float64)
        ra, rb = oracle_solution(a, solvedim), oracle_solution(b, solvedim)
        x1, v1 = shared_solve(a, solvedim, dims, buffer=buf)
        x2, _ = shared_solve(a, solvedim, dims, buffer=buf)
        assert "tmem" in v1
        assert np.array_equal(x1, x2)
        assert fwd_err(x1, ra) <= 1e-12
        xb, _ = shared_solve(b, solvedim, dims, buffer=buf)
        assert fwd_err(xb, rb) <= 1e-12, solvedim
        # a general solve scribbles over the buffer; the next shared solve is still right
        dv = to_dev(fixtures.random_dominant(dims, 5, np.float64))
        solve_dev(dv, solvedim, buffer=buf)
        xa, _ = shared_solve(a, solvedim, dims, buffer=buf)
        assert np.array_equal(xa, x1), solvedim
        # no buffer at all: no cache, same answer
        xn, vn = shared_solve(a, solvedim, dims, buffer=None)
        assert "tmem" in vn and np.array_equal(xn, x1)


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_shared_fact_ignores_out_of_range_entries(cuda, solvedim):
    dims = (24, 20, 18)
    co = shared_problem(dims, solvedim, 31, np.float64)
    ref = oracle_solution(co, solvedim)
    ax = 2 - solvedim

    def sl(i):
        s = [slice(None)] * 3
        s[ax] = i
        return tuple(s)

    for name, rows in (("ds", [0, 1]), ("dl", [0]), ("du", [-1]), ("dw", [-2, -1])):
        for r in rows:
            co[name][sl(r)] = np.nan
    got, _ = shared_solve(co, solvedim, dims)
    assert np.all(np.isfinite(got))
    assert fwd_err(got, ref) <= 1e-12


def test_shared_fact_adi_constant_coefficients_agree_with_general(cuda):
    """The ADI stencil of the 256^3 benchmark at 64^3: shared factorisation and
    the general kernels give the same field after x, y, z."""
    dims = (64, 64, 64)
    co = fixtures.adi_constant(dims)
    dg, ds_ = to_dev(co), to_dev(co)
    with ps.Handle() as h:
        for a in range(3):
            h.set_algo(a, "shared-fact")
        for axis in range(3):
            solve_dev(dg, axis)
            solve_dev(ds_, axis, handle=h)
        assert [h.kernel_that_ran(a) for a in range(3)] == ["shared-fact"] * 3
    assert fwd_err(ds_["x"].cpu().numpy(), dg["x"].cpu().numpy()) <= 1e-12


def test_shared_fact_environment_selector(cuda, monkeypatch):
    import torch

    dims = (32, 24, 16)
    co = shared_problem(dims, 1, 7, np.float64)
    ref = oracle_solution(co, 1)
    monkeypatch.setenv("PENTA_YALGO", "shared-fact")
    dv = to_dev(co)
    buf = ps.alloc_buffer(list(dims), 0, torch.float64)
    ps.gpsv_batch_legacy(*(dv[k] for k in NAMES), 1, buffer=buf)
    torch.cuda.synchronize()
    assert ps.kernel_that_ran(1) == "shared-fact"
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("dims", [(16, 8, 8), (48, 8, 8)])
def test_shared_fact_zero_pivot_is_reported(cuda, dims):
    # (16, 8, 8): the per-line kernel; (48, 8, 8): the Tensor-Memory kernel,
    # whose upper table meets the zero pivot at row 0
    co = shared_problem(dims, 0, 3, np.float64)
    co["d"][..., 0] = 0.0
    co["dl"][..., 1] = 0.0
    co["ds"][..., 2] = 0.0
    got = []
    shared_solve(co, 0, dims, check_status=False, status=got)
    st, bits = got[0]
    assert st == ps.ZERO_PIVOT and bits & 1
