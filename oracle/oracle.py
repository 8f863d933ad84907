"""ctypes front end to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product library never does.

Three CPU solvers are reachable from here:

* ``penta_oracle.c`` (``libpenta_oracle.so``): the C restatement of the
  reference's scalar solver ``src/cpu/singlenode/pentad_orig_cpu.cpp``.
* ``_ref/libpentad_orig_ref.so``: that reference file itself, compiled from the
  reference tree by ``oracle/Makefile`` (the pin for the restatement).
* ``_ref/libpentad_simd_ref.so``: the reference's OpenMP+AVX2 solver
  ``src/cpu/singlenode/pentad_cpu.cpp`` (the timed CPU baseline; it requires
  a 3-D grid with ``dims[0]`` a multiple of its vector width because it assumes a
  padded x axis, ``pentad_cpu.cpp:611-613``; see ``simd_ok``).

Arrays are numpy arrays in C order whose LAST numpy axis is the reference's
``t_dims[0]`` (the contiguous axis); ``dims`` is given fastest-first as in the
reference API.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "libpenta_oracle.so"
REF_ORIG_SO = HERE / "_ref" / "libpentad_orig_ref.so"
REF_SIMD_SO = HERE / "_ref" / "libpentad_simd_ref.so"
REF_CUDA_SO = HERE / "_ref" / "libpentad_cuda_ref.so"

#: Environment variable naming the reference source tree (read by the build
#: recipe, the fixture generator and the fixture tests); unset, the tree is
#: looked for at the path below.
REFERENCE_ENV = "PENTA_REFERENCE_DIR"
REFERENCE_DEFAULT = "/root/reference"


def reference_dir() -> Path:
    """Where the reference's sources are (they may be absent)."""
    return Path(os.environ.get(REFERENCE_ENV) or REFERENCE_DEFAULT)


_P = ctypes.c_void_p
_libs: dict[str, ctypes.CDLL] = {}


def _load(path: Path) -> ctypes.CDLL:
    key = str(path)
    if key not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (run oracle/Makefile)")
        _libs[key] = ctypes.CDLL(key)
    return _libs[key]


def _oracle() -> ctypes.CDLL:
    lib = _load(ORACLE_SO)
    if not getattr(lib, "_typed", False):
        for suf in ("d", "s"):
            f = getattr(lib, f"penta_oracle_batch_{suf}")
            f.argtypes = [_P] * 6 + [_P, ctypes.c_int, ctypes.c_int]
            f.restype = ctypes.c_int
            r = getattr(lib, f"penta_oracle_residual_{suf}")
            r.argtypes = [_P] * 7 + [_P, ctypes.c_int, ctypes.c_int]
            r.restype = ctypes.c_double
        lib.penta_oracle_fwd_err_d.argtypes = [_P, _P, ctypes.c_size_t]
        lib.penta_oracle_fwd_err_d.restype = ctypes.c_double
        lib.penta_oracle_num_threads.restype = ctypes.c_int
        lib._typed = True
    return lib


def _dims_arr(dims):
    return (ctypes.c_int * len(dims))(*[int(v) for v in dims])


def _check(arrs, dtype):
    for a in arrs:
        if a.dtype != dtype or not a.flags.c_contiguous:
            raise TypeError("oracle arrays must be C-contiguous and of one dtype")


def dims_of(a: np.ndarray) -> list[int]:
    """Reference-order dims (fastest first) of a C-order numpy array."""
    return [int(v) for v in reversed(a.shape)]


def solve(ds, dl, d, du, dw, x, solvedim, dims=None) -> np.ndarray:
    """Solve in place with the C restatement (returns ``x``)."""
    dtype = x.dtype
    _check((ds, dl, d, du, dw, x), dtype)
    dims = dims_of(x) if dims is None else list(dims)
    lib = _oracle()
    fn = lib.penta_oracle_batch_d if dtype == np.float64 else lib.penta_oracle_batch_s
    rc = fn(*(a.ctypes.data for a in (ds, dl, d, du, dw, x)), _dims_arr(dims),
            len(dims), int(solvedim))
    if rc != 0:
        raise ValueError(f"oracle rejected dims={dims} solvedim={solvedim} (rc={rc})")
    return x


def residual(ds, dl, d, du, dw, x, b, solvedim, dims=None) -> float:
    """max |A x - b| over all lines along ``solvedim``."""
    dtype = x.dtype
    _check((ds, dl, d, du, dw, x, b), dtype)
    dims = dims_of(x) if dims is None else list(dims)
    lib = _oracle()
    fn = lib.penta_oracle_residual_d if dtype == np.float64 else lib.penta_oracle_residual_s
    return float(fn(*(a.ctypes.data for a in (ds, dl, d, du, dw, x, b)),
                    _dims_arr(dims), len(dims), int(solvedim)))


def fwd_err(x: np.ndarray, ref: np.ndarray) -> float:
    """max|x - ref| / max|ref| (reference apps/fp32_accuracy_cuda.cu definition)."""
    xa = np.ascontiguousarray(x, dtype=np.float64)
    ra = np.ascontiguousarray(ref, dtype=np.float64)
    return float(_oracle().penta_oracle_fwd_err_d(xa.ctypes.data, ra.ctypes.data, xa.size))


def num_threads() -> int:
    return int(_oracle().penta_oracle_num_threads())


# --------------------------------------------------------------------------
# The reference's own compiled CPU solvers (built from the reference tree).
# --------------------------------------------------------------------------
def ref_available(which: str = "orig") -> bool:
    return {"orig": REF_ORIG_SO, "simd": REF_SIMD_SO, "cuda": REF_CUDA_SO}[which].exists()


def _ref_lib(which: str) -> ctypes.CDLL:
    path = {"orig": REF_ORIG_SO, "simd": REF_SIMD_SO, "cuda": REF_CUDA_SO}[which]
    lib = _load(path)
    if not getattr(lib, "_typed", False):
        for name in ("pentadsolver_D_gpsv_batch", "pentadsolver_S_gpsv_batch"):
            f = getattr(lib, name)
            f.argtypes = [_P] * 7 + [_P, ctypes.c_int, ctypes.c_int, _P]
            f.restype = None
        lib._typed = True
    return lib


def simd_ok(dims, dtype) -> bool:
    """Shapes the AVX2 solver handles without reading out of bounds: it assumes
    a 3-D grid whose x axis is a multiple of the vector width
    (``pentad_cpu.cpp:611-613`` pads x to SIMD_VEC = 4 in FP64, 8 in FP32)."""
    width = 4 if np.dtype(dtype) == np.float64 else 8
    return len(dims) == 3 and int(dims[0]) % width == 0


def ref_solve(ds, dl, d, du, dw, x, solvedim, which: str = "orig", dims=None):
    """Solve in place with the reference's own CPU solver ("orig" or "simd")."""
    if which not in ("orig", "simd"):
        raise ValueError("CPU reference is 'orig' or 'simd'")
    dtype = x.dtype
    _check((ds, dl, d, du, dw, x), dtype)
    dims = dims_of(x) if dims is None else list(dims)
    n = int(dims[solvedim])
    if n <= 4:
        raise ValueError("the reference solvers require sys_size > 4")
    if which == "orig" and n > 1024:
        raise ValueError("the reference scalar solver holds at most 1024 rows per system")
    if which == "simd" and not simd_ok(dims, dtype):
        raise ValueError("the reference SIMD solver needs a 3-D grid with dims[0] a "
                         "multiple of its vector width (4 FP64, 8 FP32)")
    lib = _ref_lib(which)
    fn = lib.pentadsolver_D_gpsv_batch if dtype == np.float64 else lib.pentadsolver_S_gpsv_batch
    fn(None, *(a.ctypes.data for a in (ds, dl, d, du, dw, x)), _dims_arr(dims),
       len(dims), int(solvedim), None)
    return x


def ref_cuda_solver():
    """The reference's own GPU solver (``src/cuda/singlenode/pentad_cuda.cu``
    compiled for sm_100a into ``_ref/libpentad_cuda_ref.so``), stock
    dispatch: (D_gpsv_batch taking device pointers and a device scratch
    buffer of its ``buffer_size_ext`` bytes, kernel_that_ran(direction))."""
    lib = _ref_lib("cuda")
    ran = lib.pentadsolver_kernel_that_ran
    ran.argtypes = [ctypes.c_int]
    ran.restype = ctypes.c_char_p
    return lib.pentadsolver_D_gpsv_batch, (lambda direction: ran(int(direction)).decode())


def cpu_model() -> str:
    """The host CPU's model name (``/proc/cpuinfo``), or "unknown"."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def set_threads(n: int) -> None:
    """OpenMP thread count for later oracle / reference calls in this process."""
    os.environ["OMP_NUM_THREADS"] = str(int(n))
    try:
        gomp = ctypes.CDLL("libgomp.so.1")
        gomp.omp_set_num_threads(ctypes.c_int(int(n)))
    except OSError:
        pass


# --------------------------------------------------------------------------
# The random test mesh (mesh_oracle.c) and the reference's own Mesh class
# (_ref/libmesh_ref.so, ref_mesh_shim.cpp against include/util/mesh.hpp).
# --------------------------------------------------------------------------
REF_MESH_SO = HERE / "_ref" / "libmesh_ref.so"
MESH_NAMES = ("ds", "dl", "d", "du", "dw", "x")


def mt64_nth(seed: int, n: int) -> int:
    """The n-th (1-based) output of MT19937-64 seeded with ``seed``."""
    f = _oracle().penta_oracle_mt64_nth
    f.argtypes = [ctypes.c_uint64, ctypes.c_longlong]
    f.restype = ctypes.c_uint64
    return int(f(seed, n))


def _mesh_call(fn, dims, solvedim, nthreads, dtype) -> dict:
    shape = tuple(reversed([int(v) for v in dims]))
    out = {k: np.empty(shape, dtype=dtype) for k in MESH_NAMES}
    fn.argtypes = [_P, ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_P] * 6
    fn.restype = ctypes.c_int
    rc = fn(_dims_arr(dims), len(dims), int(solvedim), int(nthreads),
            *(out[k].ctypes.data for k in MESH_NAMES))
    if rc != 0:
        raise ValueError(f"mesh generator rejected dims={dims} solvedim={solvedim}")
    return out


def mesh_random(dims, solvedim: int, nthreads: int, dtype=np.float64) -> dict:
    """The reference's random grid for ``nthreads`` OpenMP threads (restatement)."""
    suf = "d" if np.dtype(dtype) == np.float64 else "s"
    return _mesh_call(getattr(_oracle(), f"penta_oracle_mesh_random_{suf}"), dims, solvedim,
                      nthreads, dtype)


def ref_mesh_available() -> bool:
    return REF_MESH_SO.exists()


def ref_mesh_random(dims, solvedim: int, nthreads: int, dtype=np.float64) -> dict:
    """``Mesh<Float>(solvedim, dims)`` itself, run with ``nthreads`` threads."""
    suf = "d" if np.dtype(dtype) == np.float64 else "s"
    return _mesh_call(getattr(_load(REF_MESH_SO), f"ref_mesh_random_{suf}"), dims, solvedim,
                      nthreads, dtype)


def ref_mesh_load(path, dims, dtype=np.float64) -> dict:
    """``Mesh<Float>(file)`` itself: ds .. x and u of a fixture file."""
    suf = "d" if np.dtype(dtype) == np.float64 else "s"
    fn = getattr(_load(REF_MESH_SO), f"ref_mesh_load_{suf}")
    fn.argtypes = [ctypes.c_char_p] + [_P] * 7
    fn.restype = ctypes.c_int
    shape = tuple(reversed([int(v) for v in dims]))
    out = {k: np.empty(shape, dtype=dtype) for k in MESH_NAMES + ("u",)}
    fn(os.fsencode(str(path)), *(out[k].ctypes.data for k in MESH_NAMES + ("u",)))
    return out
