"""Test grids through the library's C ABI (``include/pentadsolver_mesh.h``).

The reference's tests and benchmarks get their grids from two header-only
utilities: ``Mesh<Float>(file)`` / ``DeviceMesh<Float>(file)`` read a fixture
file (``include/util/mesh.hpp:51-80``, ``include/util/device_mesh.hpp:35-50``),
and ``Mesh<Float>(solve_dim, dims)`` / ``DeviceMesh<Float>(solve_dim, dims)``
build the random benchmark grid with OpenMP threads on the host and copy it to
the GPU (``mesh.hpp:85-124``, ``device_mesh.hpp:52-65``).  Their counterparts:

* ``read_fixture`` / ``write_fixture`` / ``fixture_info``: the reference's text
  format (and a binary form of it) read and written by the library's host code;
* ``fixture_to_device``: a fixture read and uploaded, as ``DeviceMesh(file)``;
* ``random_mesh``: the random grid generated by one kernel straight into device
  arrays, bit-identical to the reference's for the same host thread count.

Array convention as in ``pentadsolver``: numpy / torch C order with the LAST
axis equal to the reference's ``dims[0]``.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

import pentadsolver as ps

TEXT, BINARY_F32, BINARY_F64 = 0, 4, 8
NAMES = ("ds", "dl", "d", "du", "dw", "x")
MAX_THREADS = 65536

_P = ctypes.c_void_p
_I = ctypes.c_int


def _fn(name, argtypes):
    f = getattr(ps.lib(), name)
    f.argtypes = argtypes
    f.restype = _I
    return f


def _prefix(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "D"
    if dt == np.float32:
        return "S"
    raise TypeError(f"unsupported dtype {dtype}")


def _check(st: int, what: str) -> None:
    if st != ps.SUCCESS:
        raise ps.PentadError(st, what)


def fixture_info(path) -> dict:
    """``{"ndims", "solvedim", "dims", "format"}`` of a fixture file."""
    nd, sd, fmt = _I(0), _I(0), _I(0)
    dims = (_I * ps.MAXDIM)()
    f = _fn("pentadsolver_fixture_info", [ctypes.c_char_p, _P, _P, _P, _P])
    _check(f(os.fsencode(path), ctypes.byref(nd), ctypes.byref(sd), dims, ctypes.byref(fmt)),
           f"fixture_info({path})")
    return {"ndims": nd.value, "solvedim": sd.value, "dims": list(dims[:nd.value]),
            "format": fmt.value}


def read_fixture(path, dtype=np.float64, with_u: bool = True) -> dict:
    """The arrays of a fixture file, parsed at ``dtype``'s precision (as
    ``Mesh<double>`` / ``Mesh<float>`` do): a dict of numpy arrays shaped
    ``reversed(dims)`` plus ``dims`` and ``solvedim``."""
    info = fixture_info(path)
    shape = tuple(reversed(info["dims"]))
    arrs = {k: np.empty(shape, dtype=dtype) for k in NAMES}
    u = np.empty(shape, dtype=dtype) if with_u else None
    f = _fn(f"pentadsolver_{_prefix(dtype)}_fixture_read", [ctypes.c_char_p] + [_P] * 7)
    _check(f(os.fsencode(path), *(arrs[k].ctypes.data for k in NAMES),
             None if u is None else u.ctypes.data), f"fixture_read({path})")
    out = dict(arrs)
    if u is not None:
        out["u"] = u
    out["dims"] = info["dims"]
    out["solvedim"] = info["solvedim"]
    return out


def write_fixture(path, arrays: dict, solvedim: int, fmt: int = TEXT) -> None:
    """Write ``arrays`` (``ds`` .. ``x`` and optionally ``u``, one dtype, numpy
    arrays whose last axis is dims[0]) as a fixture file in ``fmt``."""
    x = np.asarray(arrays["x"])
    dtype = x.dtype
    dims = [int(v) for v in reversed(x.shape)]
    cols = []
    for k in NAMES:
        a = np.ascontiguousarray(arrays[k], dtype=dtype)
        if a.shape != x.shape:
            raise ValueError("arrays must share one shape")
        cols.append(a)
    u = arrays.get("u")
    if u is not None:
        u = np.ascontiguousarray(u, dtype=dtype)
    f = _fn(f"pentadsolver_{_prefix(dtype)}_fixture_write",
            [ctypes.c_char_p, _I, _I, _I, _P] + [_P] * 7)
    cdims = (_I * len(dims))(*dims)
    _check(f(os.fsencode(path), int(fmt), len(dims), int(solvedim), cdims,
             *(a.ctypes.data for a in cols), None if u is None else u.ctypes.data),
           f"fixture_write({path})")


def fixture_to_device(path, dtype=np.float64, device="cuda") -> dict:
    """``DeviceMesh<Float>(file)``: the fixture's arrays as CUDA tensors
    (``u`` stays a host array: the reference keeps it on the host too)."""
    import torch

    fx = read_fixture(path, dtype)
    out = {k: torch.from_numpy(fx[k]).to(device) for k in NAMES}
    out["u"] = fx["u"]
    out["dims"] = fx["dims"]
    out["solvedim"] = fx["solvedim"]
    return out


def host_threads() -> int:
    """The OpenMP thread count the reference's generator would use on this
    host: the first entry of OMP_NUM_THREADS, else the CPUs this process may
    run on."""
    env = os.environ.get("OMP_NUM_THREADS", "").split(",")[0].strip()
    if env.isdigit() and int(env) > 0:
        return int(env)
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def random_mesh(dims, solvedim: int, n_threads: int | None = None, dtype=None,
                device=None, stream=None) -> dict:
    """``DeviceMesh<Float>(solvedim, dims)``: the reference's random grid for
    ``n_threads`` host threads (default ``host_threads()``), generated on the
    device into new CUDA tensors ``ds`` .. ``x`` (shape ``reversed(dims)``)."""
    import torch

    dtype = torch.float64 if dtype is None else dtype
    pre = "D" if dtype == torch.float64 else "S" if dtype == torch.float32 else None
    if pre is None:
        raise TypeError(f"unsupported dtype {dtype}")
    n_threads = host_threads() if n_threads is None else int(n_threads)
    device = torch.device("cuda" if device is None else device)
    dims = [int(v) for v in dims]
    shape = tuple(reversed(dims))
    out = {k: torch.empty(shape, dtype=dtype, device=device) for k in NAMES}
    sp = ps._stream_ptr(stream, device)
    f = _fn(f"pentadsolver_{pre}_mesh_random", [_P, _I, _I, _I] + [_P] * 6 + [_P])
    cdims = (_I * len(dims))(*dims)
    _check(f(cdims, len(dims), int(solvedim), n_threads,
             *(int(out[k].data_ptr()) for k in NAMES), sp), "mesh_random")
    out["dims"] = dims
    out["solvedim"] = int(solvedim)
    return out
