"""GPU parity: the CUDA library through its C ABI against the oracle and the
reference's golden data.

Tolerances:
  * golden fixtures: the reference's own per-element test tolerance
    (test/catch_utils.hpp:19-22): rel 1e-13 or abs 1e-15 (FP64),
    rel 1e-5 or abs 1e-6 (FP32);
  * seeded grids: forward error max|x - x_ref| / max|x_ref| <= 1e-12 (FP64)
    against the oracle and against the reference's compiled CPU solver,
    <= 1e-5 (FP32) -- the definition of apps/fp32_accuracy_cuda.cu.
"""
import os

import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import (NAMES, SELECTIONS, allclose_ref, direction, fwd_err, solve_dev,
                      to_dev)
from oracle import oracle

pytestmark = pytest.mark.gpu

FWD_TOL = {np.float64: 1e-12, np.float32: 1e-5}


def _selections_for(dirn):
    return [s for s in SELECTIONS if s[0] != "transpose" or dirn == 0]


@pytest.mark.parametrize("fam,solvedim", list(fixtures.all_fixture_cases()))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_reference_fixtures_every_kernel(cuda, fam, solvedim, dtype):
    fx = fixtures.load_fixture(fam, solvedim)
    dims = fx["dims"]
    dirn = direction(len(dims), solvedim)
    expect = fx["u"] if dtype == np.float64 else fx["u_float"]
    for label, algo, lanes in _selections_for(dirn):
        co = {k: fx[k].astype(dtype) for k in NAMES}
        dv = to_dev(co)
        with ps.Handle() as h:
            h.set_algo(dirn, algo, lanes)
            solve_dev(dv, solvedim, dims=dims, handle=h)
            ran = h.kernel_that_ran(dirn)
        got = dv["x"].cpu().numpy()
        ok, worst = allclose_ref(got, expect, dtype)
        assert ok, f"{fam} solve{solvedim} {label} ({ran}): max diff {worst:.3e}"
        want_family = {"auto": "thomas-pcr", "naive": "naive", "pcr-p1": "thomas-pcr",
                       "pcr-p2": "thomas-pcr", "transpose": "transpose"}[label]
        assert ran == want_family, (label, ran)


@pytest.mark.parametrize("name", fixtures.REFRUNS)
@pytest.mark.parametrize("tag,dtype", [("d", np.float64), ("s", np.float32)])
def test_stored_reference_runs_x_then_y_then_z(cuda, name, tag, dtype):
    z = fixtures.load_refrun(name)
    dims = [int(v) for v in z["dims"]]
    co = {k: z[f"{k}_{tag}"] for k in NAMES}
    dv = to_dev(co)
    for axis in range(3):
        solve_dev(dv, axis, dims=dims)
        got = dv["x"].cpu().numpy()
        for which in ("orig", "simd"):
            key = f"after{axis}_{which}_{tag}"
            if key in z:
                e = fwd_err(got, z[key])
                assert e <= FWD_TOL[dtype], (name, axis, which, e)
        # continue from the reference's state so errors do not compound
        dv["x"].copy_(__import__("torch").from_numpy(z[f"after{axis}_orig_{tag}"]).to("cuda"))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_config0_64cube_against_oracle_and_reference(cuda, dtype):
    dims = (64, 64, 64)
    co = fixtures.random_dominant(dims, 20240601, dtype)
    dv = to_dev(co)
    x_or = co["x"].copy()
    x_ref = co["x"].copy()
    for axis in range(3):
        solve_dev(dv, axis)
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x_or, axis)
        got = dv["x"].cpu().numpy()
        assert fwd_err(got, x_or) <= FWD_TOL[dtype], axis
        if oracle.ref_available("orig"):
            oracle.ref_solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x_ref, axis)
            assert fwd_err(got, x_ref) <= FWD_TOL[dtype], axis


ODD_DIMS = [(5,), (7,), (129,), (5, 5), (17, 6), (6, 17), (5, 7, 9), (33, 17, 6), (9, 5, 31),
            (13, 11, 7, 5), (300, 3, 2)]


@pytest.mark.parametrize("dims", ODD_DIMS)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_odd_and_ragged_shapes_every_kernel(cuda, dims, dtype):
    for solvedim in range(len(dims)):
        if dims[solvedim] <= 4:
            continue
        dirn = direction(len(dims), solvedim)
        co = fixtures.random_dominant(dims, 7 + solvedim, dtype)
        ref = co["x"].copy()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, solvedim)
        for label, algo, lanes in _selections_for(dirn):
            dv = to_dev(co)
            with ps.Handle() as h:
                h.set_algo(dirn, algo, lanes)
                solve_dev(dv, solvedim, handle=h)
            e = fwd_err(dv["x"].cpu().numpy(), ref)
            assert e <= FWD_TOL[dtype], (dims, solvedim, label, e)


@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_nan_in_ignored_entries_changes_nothing(cuda, solvedim):
    dims = (19, 12, 10)
    co = fixtures.random_dominant(dims, 31, np.float64)
    clean = {k: v.copy() for k, v in co.items()}
    fixtures.zero_out_of_range(clean, solvedim)
    dirty = {k: v.copy() for k, v in co.items()}
    ax = 2 - solvedim

    def sl(i):
        s = [slice(None)] * 3
        s[ax] = i
        return tuple(s)

    for name, rows in (("ds", [0, 1]), ("dl", [0]), ("du", [-1]), ("dw", [-2, -1])):
        for r in rows:
            dirty[name][sl(r)] = np.nan
    dirn = direction(3, solvedim)
    for label, algo, lanes in _selections_for(dirn):
        outs = []
        for c in (clean, dirty):
            dv = to_dev(c)
            with ps.Handle() as h:
                h.set_algo(dirn, algo, lanes)
                solve_dev(dv, solvedim, handle=h)
            outs.append(dv["x"].cpu().numpy())
        assert np.all(np.isfinite(outs[1])), label
        assert np.array_equal(outs[0], outs[1]), label


def test_zero_pivot_is_reported(cuda):
    dims = (16, 8, 8)
    co = fixtures.random_dominant(dims, 3, np.float64)
    co["d"][2, 3, 0] = 0.0      # first row of one x line: pivot exactly zero
    co["dl"][2, 3, 1] = 0.0
    co["ds"][2, 3, 2] = 0.0
    ps.status_check()           # clear
    dv = to_dev(co)
    solve_dev(dv, 0, check_status=False)
    st, bits = ps.status_check()
    assert st == ps.ZERO_PIVOT and bits & 1
    st, bits = ps.status_check()
    assert st == ps.SUCCESS and bits == 0


def test_naive_rejects_short_buffer(cuda):
    import torch

    dims = (16, 16, 16)
    co = fixtures.random_dominant(dims, 3, np.float64)
    dv = to_dev(co)
    small = torch.empty(1024, dtype=torch.uint8, device="cuda")
    with ps.Handle() as h:
        h.set_algo(1, "naive")
        st = ps.gpsv_batch(*(dv[k] for k in NAMES), 1, buffer=small, handle=h, check=False)
    assert st == ps.INVALID_VALUE


def test_explicit_stream_and_legacy_entry_point(cuda):
    import torch

    dims = (48, 40, 36)
    co = fixtures.random_dominant(dims, 11, np.float64)
    ref = co["x"].copy()
    for axis in range(3):
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
    dv = to_dev(co)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        for axis in range(3):
            solve_dev(dv, axis, stream=s)
    s.synchronize()
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12
    # the reference-named void entry point on the legacy default stream
    dv = to_dev(co)
    buf = ps.alloc_buffer(list(dims), 0, torch.float64)
    torch.cuda.synchronize()
    for axis in range(3):
        ps.gpsv_batch_legacy(*(dv[k] for k in NAMES), axis, buffer=buf)
    torch.cuda.synchronize()
    assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12


def test_environment_selectors_and_kernel_record(cuda, monkeypatch):
    import torch

    dims = (24, 20, 18)
    co = fixtures.random_dominant(dims, 12, np.float64)
    ref = co["x"].copy()
    for axis in range(3):
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, axis)
    cases = [
        ({"PENTA_XALGO": "naive"}, ("naive", "thomas-pcr", "thomas-pcr")),
        ({"PENTA_XALGO": "transpose", "PENTA_YZALGO": "naive"}, ("transpose", "naive", "naive")),
        ({"PENTA_YALGO": "thomas-pcr", "PENTA_YZALGO": "naive"}, ("thomas-pcr", "thomas-pcr", "naive")),
        ({"PENTA_ZALGO": "legacy"}, ("thomas-pcr", "thomas-pcr", "naive")),
        ({"PENTA_XALGO": "bogus"}, ("thomas-pcr", "thomas-pcr", "thomas-pcr")),
        ({"PENTA_PCR_LANES": "1"}, ("thomas-pcr", "thomas-pcr", "thomas-pcr")),
    ]
    for env, expect in cases:
        for k in ("PENTA_XALGO", "PENTA_YALGO", "PENTA_ZALGO", "PENTA_YZALGO", "PENTA_PCR_LANES"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        dv = to_dev(co)
        buf = ps.alloc_buffer(list(reversed(co["x"].shape)), 0, torch.float64)
        for axis in range(3):
            ps.gpsv_batch_legacy(*(dv[k] for k in NAMES), axis, buffer=buf)
        torch.cuda.synchronize()
        assert tuple(ps.kernel_that_ran(d) for d in range(3)) == expect, env
        assert fwd_err(dv["x"].cpu().numpy(), ref) <= 1e-12, env


@pytest.mark.slow
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_256cube_properties(cuda, solvedim):
    """Full-size checks at 256^3 FP64: agreement with the oracle, with the
    global-scratch kernel, and linearity in the right-hand side."""
    import torch

    dims = (256, 256, 256)
    co = fixtures.random_dominant(dims, 77, np.float64)
    ref = co["x"].copy()
    oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, solvedim)
    dv = to_dev(co)
    b = dv["x"].clone()
    solve_dev(dv, solvedim)
    x_auto = dv["x"].clone()
    assert fwd_err(x_auto.cpu().numpy(), ref) <= 1e-12
    # naive kernel agrees
    dirn = direction(3, solvedim)
    with ps.Handle() as h:
        h.set_algo(dirn, "naive")
        dv["x"].copy_(b)
        solve_dev(dv, solvedim, handle=h)
    assert fwd_err(dv["x"].cpu().numpy(), x_auto.cpu().numpy()) <= 1e-12
    # linearity: A^-1 (2 b + b') = 2 A^-1 b + A^-1 b'
    b2 = torch.from_numpy(np.random.default_rng(5).uniform(-1, 1, b.shape)).cuda()
    dv["x"].copy_(b2)
    solve_dev(dv, solvedim)
    x2 = dv["x"].clone()
    dv["x"].copy_(2 * b + b2)
    solve_dev(dv, solvedim)
    lin = (2 * x_auto + x2).cpu().numpy()
    assert fwd_err(dv["x"].cpu().numpy(), lin) <= 1e-12


def _tmem_ok(dims, solvedim, eb):
    """Shapes the Tensor-Memory kernel takes (TMA tiles when rows (x) or runs
    (y, z) are 16-byte aligned, element copies otherwise): two real rows in
    each half of the split m = R ceil(n / 2R), and its scratch for whole tiles
    of 16 lines within the reference-sized buffer.  The factor mode follows
    the m / R stages: du2, dw2 and x2 all in TMEM (up to 8 stages, no
    scratch), du2 and dw2 (16 stages), du2 alone with dw2 in the buffer (32
    stages), or all factors in the buffer."""
    n = dims[solvedim]
    inner = int(np.prod(dims[:solvedim]))
    n_sys = int(np.prod(dims)) // n
    contig = solvedim == 0
    r = 64 // eb if contig else 1024 // (16 * eb)
    aligned = True if contig else inner > 1   # misaligned grids use element copies
    mt = r * (-(-n // (2 * r)))
    stages = mt // r
    cols = r * eb // 4               # TMEM columns of one factor per stage
    cap_all = 4 if (eb == 4 and not contig) else 512 // (3 * cols) - 2
    per_row = (0 if stages <= cap_all else 1 if stages <= 512 // (2 * cols)
               else 2 if stages <= 512 // cols else 3)
    tiles = -(-n_sys // 16) if contig else (n_sys // inner) * -(-inner // 16)
    need = tiles * 2 * mt * 16 * eb * per_row
    buf = ps.buffer_size(list(dims), solvedim, eb)
    return aligned and n - mt >= 2 and need <= buf


def _x2_on_chip(dims, solvedim, eb):
    """Lines short enough that the Tensor-Memory kernel keeps x2 in TMEM too
    (up to 8 stages of R rows per half, 4 for FP32 along y/z): it needs no
    buffer at all."""
    n = dims[solvedim]
    r = 64 // eb if solvedim == 0 else 1024 // (16 * eb)
    return -(-n // (2 * r)) <= (4 if (eb == 4 and solvedim != 0) else 8)


def _old_tma_ok(dims, solvedim, eb, buffer=True):
    """Shapes the older TMA kernels take (without TMEM)."""
    n = dims[solvedim]
    inner = int(np.prod(dims[:solvedim]))
    n_sys = int(np.prod(dims)) // n
    if solvedim == 0:   # needs its (dw2, x2) scratch in a 128-byte aligned buffer
        return buffer and (n * eb) % 16 == 0 and \
            -(-n_sys // 16) * n * 32 * eb <= ps.buffer_size(list(dims), 0, eb)
    return inner > 1 and (inner * eb) % 16 == 0


def _run_chain(co, solvedim, dims, env, monkeypatch, offset=None, buffer=True):
    """One solve under the given kernel switches; returns (x, variant)."""
    import torch

    for k in ("PENTA_NO_TMA", "PENTA_NO_TMEM"):
        monkeypatch.setenv(k, "1" if k in env else "0")
    dv = to_dev(co)
    dirn = direction(len(dims), solvedim)
    with ps.Handle() as h:
        if not buffer:
            ps.gpsv_batch(*(dv[k] for k in NAMES), solvedim, buffer=None, handle=h)
            assert ps.status_check(handle=h)[1] == 0
        elif offset is not None:
            eb = dv["x"].element_size()
            need = ps.buffer_size(list(dims), solvedim, eb)
            raw = torch.empty(need + 256, dtype=torch.uint8, device="cuda")
            solve_dev(dv, solvedim, handle=h, buffer=raw[offset:offset + need])
        else:
            solve_dev(dv, solvedim, handle=h)
        var = h.variant_that_ran(dirn)
    return dv["x"].cpu().numpy(), var


CHAIN_DIMS = [(64, 64, 64), (48, 20, 33), (32, 40, 16), (20, 36, 9), (6, 40, 21),
              (34, 17, 9), (40, 21, 5), (256, 3, 2), (200, 4, 3), (300, 4, 4), (18, 5, 4)]


@pytest.mark.parametrize("dims", CHAIN_DIMS)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_kernel_chain_every_direction(cuda, dims, dtype, monkeypatch):
    """Each shape lands on the kernel its alignment and size allow -- the
    Tensor-Memory kernel, the older TMA kernels (PENTA_NO_TMEM=1) or the
    cp.async kernels (PENTA_NO_TMA=1) -- and every one agrees with the oracle.
    Buffers aligned to 16 but not 128 bytes (no L2 discards) and to 8 bytes
    only (no TMA), and no buffer at all, give the same answers."""
    co = fixtures.random_dominant(dims, 56, dtype)
    eb = np.dtype(dtype).itemsize
    tol = FWD_TOL[dtype]
    for solvedim in range(3):
        if dims[solvedim] <= 4:
            continue
        ref = {k: co[k].astype(np.float64) for k in NAMES}
        oracle.solve(ref["ds"], ref["dl"], ref["d"], ref["du"], ref["dw"], ref["x"], solvedim)
        tm, old = _tmem_ok(dims, solvedim, eb), _old_tma_ok(dims, solvedim, eb)

        def check(env, **kw):
            got, var = _run_chain(co, solvedim, dims, env, monkeypatch, **kw)
            assert fwd_err(got, ref["x"]) <= tol, (dims, solvedim, env, kw, var)
            return var

        v = check(())
        assert ("tmem" in v) == tm and (tm or ("tma" in v) == old), (solvedim, v)
        v = check(("PENTA_NO_TMEM",))
        assert "tmem" not in v and ("tma" in v) == old, (solvedim, v)
        v = check(("PENTA_NO_TMA",))
        assert "tma" not in v and "tmem" not in v, (solvedim, v)
        v = check((), offset=16)
        assert ("tmem" in v) == tm, (solvedim, v)
        # 8-byte aligned: no buffer-using TMA kernel (the strided one keeps its
        # factors on chip and still runs); lines whose factors and x2 all stay
        # in TMEM need no buffer, so the Tensor-Memory kernel runs regardless
        on_chip = tm and _x2_on_chip(dims, solvedim, eb)
        v = check((), offset=8)
        assert ("tmem" in v) == on_chip, (solvedim, v)
        assert on_chip or ("tma" in v) == (old and solvedim != 0), (solvedim, v)
        v = check((), buffer=False)
        assert ("tmem" in v) == on_chip, (solvedim, v)


LONG_DIMS = [((1040, 16, 5), 0), ((16, 1104, 5), 1), ((16, 5, 1040), 2), ((1033, 16, 5), 0),
             ((2100, 16, 5), 0), ((16, 2048, 5), 1), ((40, 1100, 5), 1)]


@pytest.mark.parametrize("dims,solvedim", LONG_DIMS)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_long_lines_factors_in_the_buffer(cuda, dims, solvedim, dtype):
    """Lines longer than Tensor Memory holds (n > 512 FP64 / 1024 FP32): the
    Tensor-Memory kernel keeps all factors in the buffer (variant "fbuf")
    and agrees with the oracle; odd n along x takes its element copies."""
    eb = np.dtype(dtype).itemsize
    co = fixtures.random_dominant(dims, 500 + solvedim, dtype)
    ref = {k: co[k].astype(np.float64) for k in NAMES}
    oracle.solve(ref["ds"], ref["dl"], ref["d"], ref["du"], ref["dw"], ref["x"], solvedim)
    dv = to_dev(co)
    with ps.Handle() as h:
        solve_dev(dv, solvedim, handle=h)
        var = h.variant_that_ran(direction(len(dims), solvedim))
    assert fwd_err(dv["x"].cpu().numpy(), ref["x"]) <= FWD_TOL[dtype], (dims, var)
    n = dims[solvedim]
    long_line = n > (512 if eb == 8 else 1024)
    if _tmem_ok(dims, solvedim, eb):
        assert "tmem" in var and (("fbuf" in var) == long_line), (dims, var)


# Odd extents along every axis, partial tiles of 16 lines, and element counts
# whose last 16-byte chunk is partial (the bulk windows at the array's end take
# their last elements with plain loads).
MISALIGNED_DIMS = [(33, 17, 9), (255, 7, 5), (17, 255, 3), (9, 7, 255), (50, 13, 7),
                   (31, 31, 31), (66, 34, 18), (129, 3, 65)]


def _loads_run(co, solvedim, loads, monkeypatch):
    monkeypatch.setenv("PENTA_TMEM_LOADS", loads)   # "" = the default choice
    dv = to_dev(co)
    dirn = direction(3, solvedim)
    with ps.Handle() as h:
        solve_dev(dv, solvedim, handle=h)
        var = h.variant_that_ran(dirn)
    monkeypatch.delenv("PENTA_TMEM_LOADS")
    return dv["x"].cpu().numpy(), var


@pytest.mark.parametrize("dims", MISALIGNED_DIMS)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_misaligned_grids_bulk_element_and_tma_loads_agree(cuda, dims, dtype, monkeypatch):
    """Rows (x) or runs (y, z) that do not start on 16-byte boundaries: the
    Tensor-Memory kernel fetches them by 16-byte cp.async copies of aligned
    supersets (default), by element copies (PENTA_TMEM_LOADS=element), as TMA
    boxes of a group view (=group: pairs or quadruples of rows / lines are
    16-byte periodic; the ones outside whole groups by bulk copies), or all by
    bulk copies of aligned supersets (=bulk); aligned rows and runs by TMA
    tiles.  The same arithmetic runs on the same values
    whichever way they arrive, so the results are identical bit for bit, and
    equal the oracle's."""
    eb = np.dtype(dtype).itemsize
    co = fixtures.random_dominant(dims, 91, dtype)
    for solvedim in range(3):
        n = dims[solvedim]
        inner = int(np.prod(dims[:solvedim]))
        if n <= 4 or not _tmem_ok(dims, solvedim, eb):
            continue
        aligned = ((n if solvedim == 0 else inner) * eb) % 16 == 0
        ref = co["x"].copy()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], ref, solvedim)
        x_auto, v_auto = _loads_run(co, solvedim, "", monkeypatch)
        x_grp, v_grp = _loads_run(co, solvedim, "group", monkeypatch)
        x_bulk, v_bulk = _loads_run(co, solvedim, "bulk", monkeypatch)
        x_elm, v_elm = _loads_run(co, solvedim, "element", monkeypatch)
        assert "chunk" not in v_elm and "grp" not in v_elm and "bulk" not in v_elm, v_elm
        assert np.array_equal(x_auto.view(np.uint8), x_elm.view(np.uint8)), (dims, solvedim)
        assert "tmem" in v_auto and "tmem" in v_grp and "tmem" in v_bulk
        assert ("chunk" in v_auto) == (not aligned), (dims, solvedim, v_auto)
        assert ("grp" in v_grp) == (not aligned), (dims, solvedim, v_grp)
        assert "bulk" in v_bulk, v_bulk
        assert fwd_err(x_auto, ref) <= FWD_TOL[dtype], (dims, solvedim, v_auto)
        assert np.array_equal(x_auto.view(np.uint8), x_grp.view(np.uint8)), (dims, solvedim)
        assert np.array_equal(x_auto.view(np.uint8), x_bulk.view(np.uint8)), (dims, solvedim)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_bulk_loads_on_aligned_grids_equal_tma_tiles(cuda, dtype, monkeypatch):
    for dims in ((64, 48, 40), (256, 16, 8), (16, 20, 512)):
        co = fixtures.random_dominant(dims, 17, dtype)
        for solvedim in range(3):
            if not _tmem_ok(dims, solvedim, np.dtype(dtype).itemsize):
                continue
            x_tma, v_tma = _loads_run(co, solvedim, "", monkeypatch)
            x_bulk, v_bulk = _loads_run(co, solvedim, "bulk", monkeypatch)
            assert "tmem" in v_tma and "bulk" not in v_tma and "bulk" in v_bulk, (v_tma, v_bulk)
            assert np.array_equal(x_tma.view(np.uint8), x_bulk.view(np.uint8)), (dims, solvedim)


# x lines whose halves take an odd number of stages: the last step of every tile
# leaves through the shared output buffer without a partner step, and the next
# tile must not write that buffer while its store may still be reading it
ODD_STAGE_X = [((24, 300, 40), np.float32),   # 1 stage (16 rows a stage), all in TMEM
               ((40, 300, 40), np.float64),   # 3 stages (8 rows), all in TMEM
               ((200, 100, 20), np.float64),  # 13 stages, x2 through the buffer
               ((400, 60, 20), np.float32)]   # 13 stages


@pytest.mark.parametrize("dims,dtype", ODD_STAGE_X)
def test_x_tiles_with_an_odd_number_of_stages(cuda, dims, dtype):
    co = fixtures.random_dominant(dims, 91, dtype)
    ref = {k: co[k].astype(np.float64) for k in NAMES}
    oracle.solve(ref["ds"], ref["dl"], ref["d"], ref["du"], ref["dw"], ref["x"], 0)
    for _ in range(5):
        dv = to_dev(co)
        solve_dev(dv, 0)
        assert fwd_err(dv["x"].cpu().numpy(), ref["x"]) <= FWD_TOL[dtype], dims
