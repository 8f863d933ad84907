"""The oracle pinned against the reference (CPU only).

* The C restatement reproduces the reference's golden fixtures
  (test/gen_testcases.py output; tolerances of test/catch_utils.hpp:19-22).
* It is bit-identical to the reference's own scalar solver compiled from the
  reference tree (oracle/_ref), and agrees with the stored reference runs.
* The math contract: out-of-range couplings are ignored whatever they hold.
"""
import numpy as np
import pytest

import fixtures
from oracle import oracle

# test/catch_utils.hpp:19-22 (per element: rel OR abs)
TOL = {np.float64: (1e-13, 1e-15), np.float32: (1e-5, 1e-6)}


def allclose_ref(actual, expected, dtype):
    rel, ab = TOL[dtype]
    diff = np.abs(actual.astype(np.float64) - expected.astype(np.float64))
    ok = (diff <= ab) | (diff <= rel * np.abs(expected.astype(np.float64)))
    return bool(np.all(ok)), float(diff.max())


@pytest.mark.parametrize("fam,solvedim", list(fixtures.all_fixture_cases()))
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_matches_reference_fixtures(fam, solvedim, dtype):
    fx = fixtures.load_fixture(fam, solvedim)
    arrs = [np.ascontiguousarray(fx[k].astype(dtype)) for k in ("ds", "dl", "d", "du", "dw", "x")]
    oracle.solve(*arrs, solvedim, dims=fx["dims"])
    expect = fx["u"] if dtype == np.float64 else fx["u_float"]
    ok, worst = allclose_ref(arrs[5], expect, dtype)
    assert ok, f"{fam} solve{solvedim} {dtype.__name__}: max diff {worst:.3e}"


def test_fixture_rotation_matches_generator_layout():
    # solvedim-k fixtures are the generator's axis rotation of solvedim 0
    base = fixtures.load_family("three_dim_large")
    f1 = fixtures.rotate(base, 1)
    assert f1["dims"] == [32, 32, 32] and f1["solvedim"] == 1
    # a line along reference dim 1 of f1 is a line along dim 0 of the base
    assert np.array_equal(f1["x"][3, :, 5], base["x"][5, 3, :])


@pytest.mark.parametrize("name", fixtures.REFRUNS)
@pytest.mark.parametrize("tag,dtype", [("d", np.float64), ("s", np.float32)])
def test_oracle_reproduces_stored_reference_runs(name, tag, dtype):
    z = fixtures.load_refrun(name)
    dims = [int(v) for v in z["dims"]]
    co = {k: z[f"{k}_{tag}"].copy() for k in ("ds", "dl", "d", "du", "dw", "x")}
    x = co["x"]
    for axis in range(3):
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x, axis, dims=dims)
        assert np.array_equal(x, z[f"after{axis}_orig_{tag}"]), (name, axis)
        if f"after{axis}_simd_{tag}" in z:
            ref = z[f"after{axis}_simd_{tag}"]
            assert oracle.fwd_err(x, ref) < (1e-14 if tag == "d" else 1e-5)


@pytest.mark.skipif(not oracle.ref_available("orig"), reason="oracle/_ref not built")
@pytest.mark.parametrize("dims", [(24, 10, 7), (7, 33, 5), (5, 5, 5), (64,), (17, 9)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_bit_identical_to_compiled_reference(dims, dtype):
    for axis in range(len(dims)):
        if dims[axis] <= 4:
            continue
        co = fixtures.random_dominant(dims, 99 + axis, dtype)
        x1 = co["x"].copy()
        x2 = co["x"].copy()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x1, axis)
        oracle.ref_solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x2, axis)
        assert np.array_equal(x1, x2), (dims, axis)


@pytest.mark.parametrize("axis", [0, 1, 2])
def test_out_of_range_couplings_are_ignored(axis):
    dims = (11, 9, 8)
    co = fixtures.random_dominant(dims, 5, np.float64)
    clean = {k: v.copy() for k, v in co.items()}
    fixtures.zero_out_of_range(clean, axis)
    x_clean = clean["x"].copy()
    oracle.solve(clean["ds"], clean["dl"], clean["d"], clean["du"], clean["dw"], x_clean, axis)
    # poison exactly the entries every solver must ignore
    dirty = {k: v.copy() for k, v in co.items()}
    nd = 3
    ax = nd - 1 - axis

    def sl(i):
        s = [slice(None)] * nd
        s[ax] = i
        return tuple(s)

    for name, rows in (("ds", [0, 1]), ("dl", [0]), ("du", [-1]), ("dw", [-2, -1])):
        for r in rows:
            dirty[name][sl(r)] = np.nan
    x_dirty = dirty["x"].copy()
    oracle.solve(dirty["ds"], dirty["dl"], dirty["d"], dirty["du"], dirty["dw"], x_dirty, axis)
    assert np.array_equal(x_clean, x_dirty)


def test_oracle_residual_small_on_config0_shape():
    dims = (64, 64, 64)
    co = fixtures.random_dominant(dims, 2024, np.float64)
    for axis in range(3):
        b = co["x"].copy()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], co["x"], axis)
        r = oracle.residual(co["ds"], co["dl"], co["d"], co["du"], co["dw"], co["x"], b, axis)
        assert r < 1e-13


def test_oracle_rejects_bad_shapes():
    a = np.zeros((4, 4), dtype=np.float64)
    with pytest.raises(ValueError):
        oracle.solve(a, a, a, a, a, a.copy(), 2)
