"""Test grids without a GPU: the random-mesh oracle and fixture I/O.

* The oracle's MT19937-64 gives the C++ standard's known answer, and its
  random mesh is bit-identical to the reference's own ``Mesh<Float>(solve_dim,
  dims)`` (``include/util/mesh.hpp:85-124``, compiled into
  ``oracle/_ref/libmesh_ref.so``) for several shapes and thread counts.
* The library's fixture reader gives, for every golden fixture written out in
  the reference's text layout (``test/gen_testcases.py:50-79``), exactly the
  values ``Mesh<double>(file)`` / ``Mesh<float>(file)`` read
  (``mesh.hpp:51-80``); the reference's shipped files too when the reference
  tree is present.
* Text and binary files round-trip bit-exactly; malformed files are errors
  that write nothing.  All of this is host code: no device is touched.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import fixtures
import mesh
import pentadsolver as ps
from oracle import oracle

SHIPPED = oracle.reference_dir() / "test" / "cpu" / "singlenode" / "files"

needs_ref = pytest.mark.skipif(not oracle.ref_mesh_available(),
                               reason="oracle/_ref/libmesh_ref.so not built")


def same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    return a.dtype == b.dtype and a.shape == b.shape and \
        np.array_equal(np.ascontiguousarray(a).view(np.uint8),
                       np.ascontiguousarray(b).view(np.uint8))


def test_mt19937_64_known_answer():
    # C++ [rand.predef]: the 10000th output of a default-constructed
    # mt19937_64 (seed 5489) is 9981545732273789042.
    assert oracle.mt64_nth(5489, 10000) == 9981545732273789042


MESH_CASES = [((5,), 0), ((9, 7), 0), ((9, 7), 1), ((16, 9, 5), 0), ((16, 9, 5), 1),
              ((16, 9, 5), 2), ((33, 17, 4), 1), ((1, 4, 3), 0), ((2, 5, 3), 0),
              ((3, 1, 2), 1), ((1, 1, 1), 2), ((40, 3, 30), 2)]


@needs_ref
@pytest.mark.parametrize("dims,solvedim", MESH_CASES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_mesh_oracle_is_the_reference_generator(dims, solvedim, dtype):
    for threads in (1, 3, 8, 64):
        got = oracle.mesh_random(dims, solvedim, threads, dtype)
        want = oracle.ref_mesh_random(dims, solvedim, threads, dtype)
        for k in oracle.MESH_NAMES:
            assert same_bits(got[k], want[k]), (dims, solvedim, threads, k)


def test_mesh_depends_on_the_thread_count():
    a = oracle.mesh_random((8, 8, 8), 0, 1)
    b = oracle.mesh_random((8, 8, 8), 0, 2)
    # thread 0's chunk starts the same; the second half comes from another stream
    assert same_bits(a["d"][:4], b["d"][:4])
    assert not np.array_equal(a["d"][4:], b["d"][4:])


def reference_text(fx: dict) -> str:
    """A fixture in the layout test/gen_testcases.py writes: Python's str() of
    every stored value reproduces the reference generator's tokens."""
    lines = [f"{len(fx['dims'])} {fx['solvedim']}", " ".join(str(v) for v in fx["dims"])]
    for k in ("ds", "dl", "d", "du", "dw", "x", "u", "u_float"):
        lines.append(" ".join(str(float(v)) for v in fx[k].ravel()))
    return "\n".join(lines) + "\n"


FIXTURE_CASES = [(fam, k) for fam, nd in fixtures.FAMILIES.items() for k in range(nd)]


@pytest.mark.parametrize("fam,solvedim", FIXTURE_CASES)
def test_text_fixture_reads_as_the_reference(tmp_path, fam, solvedim):
    fx = fixtures.load_fixture(fam, solvedim)
    path = tmp_path / f"{fam}_solve{solvedim}"
    path.write_text(reference_text(fx))
    info = mesh.fixture_info(path)
    assert info == {"ndims": len(fx["dims"]), "solvedim": solvedim, "dims": fx["dims"],
                    "format": mesh.TEXT}
    d64 = mesh.read_fixture(path, np.float64)
    for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
        assert same_bits(d64[k], fx[k]), k
    s32 = mesh.read_fixture(path, np.float32)
    # FP32 values are parsed from the text (strtof), u from the FP32 line
    for k in ("ds", "dl", "d", "du", "dw", "x"):
        assert np.max(np.abs(s32[k].astype(np.float64) - fx[k])) <= \
            np.max(np.abs(fx[k])) * 2.0 ** -24
    assert np.max(np.abs(s32["u"].astype(np.float64) - fx["u_float"])) <= \
        np.max(np.abs(fx["u_float"])) * 2.0 ** -24
    if oracle.ref_mesh_available():
        for dtype, got in ((np.float64, d64), (np.float32, s32)):
            want = oracle.ref_mesh_load(path, fx["dims"], dtype)
            for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
                assert same_bits(got[k], want[k]), (dtype, k)


@needs_ref
@pytest.mark.skipif(not SHIPPED.is_dir(), reason="reference tree not present")
def test_shipped_reference_files_read_as_the_reference():
    files = sorted(p for p in SHIPPED.iterdir() if p.is_file())
    assert files
    for path in files:
        info = mesh.fixture_info(path)
        for dtype in (np.float64, np.float32):
            got = mesh.read_fixture(path, dtype)
            want = oracle.ref_mesh_load(path, info["dims"], dtype)
            for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
                assert same_bits(got[k], want[k]), (path.name, dtype, k)


def random_arrays(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
        a = rng.standard_normal(shape) * 10.0 ** rng.integers(-30, 30, shape)
        out[k] = a.astype(dtype)
    # exact zeros, negative zero, a subnormal and extremes survive the trip
    info = np.finfo(dtype)
    out["ds"].ravel()[:5] = [0.0, -0.0, info.tiny / 4, info.max, -info.max]
    return out


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("fmt", ["text", "binary"])
def test_round_trip(tmp_path, dtype, fmt):
    arrs = random_arrays((3, 5, 7), dtype, 5)
    code = mesh.TEXT if fmt == "text" else (mesh.BINARY_F64 if dtype == np.float64
                                            else mesh.BINARY_F32)
    path = tmp_path / "grid.fx"
    mesh.write_fixture(path, arrs, solvedim=2, fmt=code)
    info = mesh.fixture_info(path)
    assert info == {"ndims": 3, "solvedim": 2, "dims": [7, 5, 3], "format": code}
    back = mesh.read_fixture(path, dtype)
    for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
        assert same_bits(back[k], arrs[k]), k


def test_text_written_by_the_library_reads_in_the_reference(tmp_path):
    if not oracle.ref_mesh_available():
        pytest.skip("oracle/_ref/libmesh_ref.so not built")
    # values inside FP32's range: Mesh<float> stops reading at an overflow
    rng = np.random.default_rng(9)
    arrs = {k: rng.standard_normal((4, 6)) * 10.0 ** rng.integers(-30, 30, (4, 6))
            for k in ("ds", "dl", "d", "du", "dw", "x", "u")}
    path = tmp_path / "grid.txt"
    mesh.write_fixture(path, arrs, solvedim=1)
    want = oracle.ref_mesh_load(path, [6, 4], np.float64)
    for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
        assert same_bits(want[k], arrs[k]), k
    want32 = oracle.ref_mesh_load(path, [6, 4], np.float32)
    assert same_bits(want32["u"], arrs["u"].astype(np.float32))


def test_binary_without_u(tmp_path):
    arrs = random_arrays((2, 6), np.float32, 3)
    del arrs["u"]
    path = tmp_path / "nou.fx"
    mesh.write_fixture(path, arrs, solvedim=0, fmt=mesh.BINARY_F32)
    back = mesh.read_fixture(path, np.float32, with_u=False)
    assert same_bits(back["x"], arrs["x"])
    with pytest.raises(ps.PentadError):
        mesh.read_fixture(path, np.float32, with_u=True)


def test_malformed_files_are_errors_that_write_nothing(tmp_path):
    fx = fixtures.load_fixture("two_dim_small", 0)
    good = reference_text(fx)
    cases = {
        "missing": None,
        "short": good[: len(good) // 2],
        "word": good.replace(str(float(fx["d"].ravel()[3])), "abc", 1),
        "ndims": "9 0\n" + "1 " * 9 + "\n",
        "solvedim": "2 2\n5 5\n",
        "empty": "",
        "nan": good.replace(str(float(fx["d"].ravel()[3])), "nan", 1),
        "hex": good.replace(str(float(fx["d"].ravel()[3])), "0x1p3", 1),
    }
    for name, text in cases.items():
        path = tmp_path / name
        if text is not None:
            path.write_text(text)
        with pytest.raises(ps.PentadError) as e:
            mesh.fixture_info(path) if name in ("missing", "ndims", "solvedim", "empty") \
                else mesh.read_fixture(path, np.float64)
        assert e.value.status == ps.INVALID_VALUE, name
    # a failed read leaves the destination as it was
    import ctypes
    path = tmp_path / "short"
    n = int(np.prod(fx["dims"]))
    dst = [np.full(n, 7.0) for _ in range(7)]
    f = ps.lib().pentadsolver_D_fixture_read
    f.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 7
    f.restype = ctypes.c_int
    assert f(str(path).encode(), *(a.ctypes.data for a in dst)) == ps.INVALID_VALUE
    assert all((a == 7.0).all() for a in dst)
    # a binary file of the other precision
    arrs = random_arrays((2, 5), np.float64, 1)
    path = tmp_path / "f64.fx"
    mesh.write_fixture(path, arrs, 0, mesh.BINARY_F64)
    with pytest.raises(ps.PentadError):
        mesh.read_fixture(path, np.float32)
    # a text value beyond FP32's range: an error for the FP32 reader only
    text = tmp_path / "big.txt"
    big = dict(arrs)
    big["d"] = arrs["d"].copy()
    big["d"][0, 0] = 1e300
    mesh.write_fixture(text, big, 0)
    assert mesh.read_fixture(text, np.float64)["d"][0, 0] == 1e300
    with pytest.raises(ps.PentadError):
        mesh.read_fixture(text, np.float32)


def test_mesh_random_rejects_bad_arguments_without_a_device():
    import ctypes
    f = ps.lib().pentadsolver_D_mesh_random
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int] + \
        [ctypes.c_void_p] * 7
    f.restype = ctypes.c_int
    dims = (ctypes.c_int * 3)(8, 8, 8)
    fake = [ctypes.c_void_p(256)] * 6
    for nd, sd, nt in ((3, 3, 4), (0, 0, 4), (3, 0, 0), (3, 0, mesh.MAX_THREADS + 1)):
        assert f(dims, nd, sd, nt, *fake, None) == ps.INVALID_VALUE
    bad = (ctypes.c_int * 3)(8, 0, 8)
    assert f(bad, 3, 0, 4, *fake, None) == ps.INVALID_VALUE
    assert f(dims, 3, 0, 4, None, *fake[1:], None) == ps.INVALID_VALUE


@pytest.mark.parametrize("shape", [(7,), (2, 1, 3, 1, 2, 1, 2, 2)])
@pytest.mark.parametrize("fmt", ["text", "binary"])
def test_round_trip_any_rank(tmp_path, shape, fmt):
    arrs = random_arrays(shape, np.float64, 11)
    code = mesh.TEXT if fmt == "text" else mesh.BINARY_F64
    path = tmp_path / "grid.fx"
    mesh.write_fixture(path, arrs, solvedim=len(shape) - 1, fmt=code)
    info = mesh.fixture_info(path)
    assert info["ndims"] == len(shape) and info["dims"] == list(reversed(shape))
    assert info["solvedim"] == len(shape) - 1 and info["format"] == code
    back = mesh.read_fixture(path, np.float64)
    for k in ("ds", "dl", "d", "du", "dw", "x", "u"):
        assert same_bits(back[k], arrs[k]), k
