"""Python front end to libpentadsolver_b200.so through its C ABI (ctypes).

Mirrors the reference's interface for the path (include/pentadsolver.hpp):
``gpsv_batch`` takes the five diagonals and the in/out right-hand side as
device arrays of one grid, the solve dimension, and a caller-owned scratch
buffer of ``buffer_size`` bytes.  Arrays are torch CUDA tensors in C order
whose last axis is the reference's ``t_dims[0]`` (the contiguous x axis);
``dims`` are derived fastest-first exactly as the reference API takes them.

There is no CPU fallback: every call goes to the CUDA library, and loading
fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpentadsolver_b200.so"

SUCCESS = 0
NOT_INITIALIZED = 1
ALLOC_FAILED = 2
INVALID_VALUE = 3
EXECUTION_FAILED = 6
INTERNAL_ERROR = 7
ZERO_PIVOT = 9

DIR_X, DIR_MIDDLE, DIR_OUTERMOST = 0, 1, 2

_P = ctypes.c_void_p
_I = ctypes.c_int
_Z = ctypes.c_size_t
_lib = None


class PentadError(RuntimeError):
    def __init__(self, status: int, what: str):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})")


def lib() -> ctypes.CDLL:
    """Load (once) and type the shared library."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {HERE}`")
    L = ctypes.CDLL(str(LIB_PATH))
    L.pentadsolver_create.argtypes = [ctypes.POINTER(_P), _P, _I, _P]
    L.pentadsolver_create.restype = None
    L.pentadsolver_destroy.argtypes = [ctypes.POINTER(_P)]
    L.pentadsolver_destroy.restype = None
    for pre in ("D", "S"):
        f = getattr(L, f"pentadsolver_{pre}_gpsv_batch_buffer_size_ext")
        f.argtypes = [_P] * 7 + [_P, _I, _I]
        f.restype = _Z
        f = getattr(L, f"pentadsolver_{pre}_gpsv_batch")
        f.argtypes = [_P] * 7 + [_P, _I, _I, _P]
        f.restype = None
        f = getattr(L, f"pentadsolver_{pre}_gpsv_batch_ex")
        f.argtypes = [_P] * 7 + [_P, _I, _I, _P, _Z, _P]
        f.restype = _I
        f = getattr(L, f"pentadsolver_{pre}_gpsv_batch_two_buffer")
        f.argtypes = [_P] * 7 + [_P, _I, _I, _P, _P]
        f.restype = None
        f = getattr(L, f"pentadsolver_{pre}_gpsv_batch_buffer_size_two_buffer")
        f.argtypes = [_P] * 7 + [_P, _I, _I, ctypes.POINTER(_Z), ctypes.POINTER(_Z)]
        f.restype = None
    L.pentadsolver_kernel_that_ran.argtypes = [_I]
    L.pentadsolver_kernel_that_ran.restype = ctypes.c_char_p
    L.pentadsolver_kernel_that_ran_ex.argtypes = [_P, _I]
    L.pentadsolver_kernel_that_ran_ex.restype = ctypes.c_char_p
    L.pentadsolver_variant_that_ran.argtypes = [_P, _I]
    L.pentadsolver_variant_that_ran.restype = ctypes.c_char_p
    L.pentadsolver_buffer_size_ex.argtypes = [_P, _I, _P, _I, _I, ctypes.POINTER(_Z)]
    L.pentadsolver_buffer_size_ex.restype = _I
    L.pentadsolver_status_check.argtypes = [_P, _P, ctypes.POINTER(_I)]
    L.pentadsolver_status_check.restype = _I
    L.pentadsolver_set_algo.argtypes = [_P, _I, ctypes.c_char_p, _I]
    L.pentadsolver_set_algo.restype = _I
    L.pentadsolver_status_string.argtypes = [_I]
    L.pentadsolver_status_string.restype = ctypes.c_char_p
    _lib = L
    return L


def status_string(status: int) -> str:
    return lib().pentadsolver_status_string(int(status)).decode()


def _dims(dims):
    return (ctypes.c_int * len(dims))(*[int(v) for v in dims])


def dims_of(t) -> list[int]:
    """Reference-order dims (fastest first) of a C-order array."""
    return [int(v) for v in reversed(tuple(t.shape))]


def _elem_prefix(dtype) -> tuple[str, int]:
    s = str(dtype)
    if s.endswith("float64"):
        return "D", 8
    if s.endswith("float32"):
        return "S", 4
    raise TypeError(f"unsupported dtype {dtype}: float64 or float32")


class Handle:
    """A library context (``pentadsolver_create`` / ``pentadsolver_destroy``)."""

    def __init__(self):
        self._h = _P()
        lib().pentadsolver_create(ctypes.byref(self._h), None, 0, None)

    @property
    def value(self):
        return self._h

    def close(self):
        if self._h:
            lib().pentadsolver_destroy(ctypes.byref(self._h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_algo(self, direction: int, algo: str | None, pcr_lanes: int = 0) -> None:
        st = lib().pentadsolver_set_algo(self._h, int(direction),
                                         None if algo is None else algo.encode(),
                                         int(pcr_lanes))
        if st != SUCCESS:
            raise PentadError(st, "set_algo")

    def kernel_that_ran(self, direction: int) -> str:
        return lib().pentadsolver_kernel_that_ran_ex(self._h, int(direction)).decode()

    def variant_that_ran(self, direction: int) -> str:
        return lib().pentadsolver_variant_that_ran(self._h, int(direction)).decode()


def _hval(handle):
    if handle is None:
        return None
    return handle.value if isinstance(handle, Handle) else handle


def buffer_size(dims, solvedim: int, elem_bytes: int = 8, handle=None) -> int:
    out = ctypes.c_size_t(0)
    st = lib().pentadsolver_buffer_size_ex(_hval(handle), int(elem_bytes), _dims(dims),
                                           len(dims), int(solvedim), ctypes.byref(out))
    if st != SUCCESS:
        raise PentadError(st, "buffer_size")
    return int(out.value)


def kernel_that_ran(direction: int) -> str:
    return lib().pentadsolver_kernel_that_ran(int(direction)).decode()


def _ptr(t) -> int:
    return int(t.data_ptr())


def _check_arrays(arrs):
    x = arrs[-1]
    for a in arrs:
        if not a.is_cuda or not a.is_contiguous():
            raise ValueError("arrays must be contiguous CUDA tensors")
        if a.dtype != x.dtype or tuple(a.shape) != tuple(x.shape):
            raise ValueError("arrays must share dtype and shape")


def gpsv_batch(ds, dl, d, du, dw, x, solvedim: int, buffer=None, stream=None,
               handle=None, dims=None, check: bool = True) -> int:
    """Solve in place along ``solvedim`` (``pentadsolver_{D,S}_gpsv_batch_ex``).

    ``buffer`` is a CUDA tensor used as scratch (any dtype); ``stream`` a
    ``torch.cuda.Stream`` or raw handle (default: torch's current stream).
    Returns the status; raises on failure when ``check``.
    """
    import torch

    _check_arrays((ds, dl, d, du, dw, x))
    pre, _ = _elem_prefix(x.dtype)
    dims = dims_of(x) if dims is None else list(dims)
    if stream is None:
        stream = torch.cuda.current_stream(x.device)
    sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    bptr, bbytes = (None, 0) if buffer is None else (_ptr(buffer),
                                                     buffer.numel() * buffer.element_size())
    fn = getattr(lib(), f"pentadsolver_{pre}_gpsv_batch_ex")
    st = fn(_hval(handle), *(_ptr(a) for a in (ds, dl, d, du, dw, x)), _dims(dims),
            len(dims), int(solvedim), bptr, bbytes, sp)
    if check and st != SUCCESS:
        raise PentadError(st, "gpsv_batch")
    return st


def gpsv_batch_legacy(ds, dl, d, du, dw, x, solvedim: int, buffer=None, handle=None,
                      dims=None) -> None:
    """The reference-named void entry point ``pentadsolver_{D,S}_gpsv_batch``
    (legacy default stream, errors on stderr)."""
    _check_arrays((ds, dl, d, du, dw, x))
    pre, _ = _elem_prefix(x.dtype)
    dims = dims_of(x) if dims is None else list(dims)
    fn = getattr(lib(), f"pentadsolver_{pre}_gpsv_batch")
    fn(_hval(handle), *(_ptr(a) for a in (ds, dl, d, du, dw, x)), _dims(dims), len(dims),
       int(solvedim), None if buffer is None else _ptr(buffer))


#: status bits (pentadsolver_status_check)
ZERO_PIVOT_BIT = 1
TIMEOUT_BIT = 2


def status_check(stream=None, handle=None) -> tuple[int, int]:
    """Read and clear the status bits of ``handle``'s solves (the NULL
    handle's shared word when None), then synchronise: (status, bits)."""
    sp = None
    if stream is not None:
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    bits = ctypes.c_int(0)
    st = lib().pentadsolver_status_check(_hval(handle), sp, ctypes.byref(bits))
    return int(st), int(bits.value)


def selftest_bounded_wait(limit_us: int, stream=None, handle=None) -> int:
    """Launch the kernel whose one wait never completes; it gives up after
    ``limit_us`` and raises TIMEOUT_BIT in the handle's status word."""
    sp = None
    if stream is not None:
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    return int(_typed("pentadsolver_selftest_bounded_wait", [_P, ctypes.c_uint, _P])(
        _hval(handle), int(limit_us), sp))


def alloc_buffer(dims, solvedim: int, dtype, device="cuda"):
    """A scratch tensor of ``buffer_size`` bytes (the caller owns scratch)."""
    import torch

    _, eb = _elem_prefix(dtype)
    nbytes = max(buffer_size(dims, solvedim, eb), 256)
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def library_loaded_path() -> str:
    return os.fspath(LIB_PATH)


# ---------------------------------------------------------------------------
# Plans (many grids, one persistent launch) and mixed-precision refinement
# ---------------------------------------------------------------------------
MAXDIM = 8


class GridDesc(ctypes.Structure):
    """pentadsolver_grid_t"""
    _fields_ = [("ds", _P), ("dl", _P), ("d", _P), ("du", _P), ("dw", _P), ("x", _P),
                ("ndim", _I), ("dims", _I * MAXDIM)]


def _grid_descs(grids):
    """grids: sequence of dicts with the six tensors ds, dl, d, du, dw, x."""
    arr = (GridDesc * len(grids))()
    for i, g in enumerate(grids):
        _check_arrays([g[k] for k in ("ds", "dl", "d", "du", "dw", "x")])
        dims = dims_of(g["x"])
        arr[i].ds, arr[i].dl, arr[i].d = _ptr(g["ds"]), _ptr(g["dl"]), _ptr(g["d"])
        arr[i].du, arr[i].dw, arr[i].x = _ptr(g["du"]), _ptr(g["dw"]), _ptr(g["x"])
        arr[i].ndim = len(dims)
        for k, v in enumerate(dims):
            arr[i].dims[k] = v
    return arr


def _typed(name, argtypes, restype=_I):
    f = getattr(lib(), name)
    f.argtypes = argtypes
    f.restype = restype
    return f


def _stream_ptr(stream, device):
    import torch

    if stream is None:
        stream = torch.cuda.current_stream(device)
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream


class Plan:
    """A fixed set of grids solved along ``solvedim`` by one persistent launch
    (``pentadsolver_plan_create`` / ``_execute``).  ``refine_steps`` (FP64
    grids only) makes it a mixed-precision plan: FP32 sweeps plus that many
    FP64 residual/correction rounds.  The plan keeps references to the grids'
    tensors and owns its buffer; execute() is capturable in a CUDA graph."""

    def __init__(self, grids, solvedim: int, refine_steps: int | None = None, ctas: int = 0,
                 handle=None, scratch=None):
        import torch

        self.grids = list(grids)
        self.solvedim = int(solvedim)
        self.refine = refine_steps is not None
        self._descs = _grid_descs(self.grids)
        x0 = self.grids[0]["x"]
        self.device = x0.device
        eb = x0.element_size()
        n = len(self.grids)
        size = ctypes.c_size_t(0)
        if self.refine:
            if x0.dtype != torch.float64:
                raise ValueError("refinement plans take FP64 grids")
            st = _typed("pentadsolver_refine_plan_buffer_size",
                        [_P, _I, ctypes.POINTER(GridDesc), _I, ctypes.POINTER(_Z)])(
                _hval(handle), n, self._descs, self.solvedim, ctypes.byref(size))
        else:
            st = _typed("pentadsolver_plan_buffer_size",
                        [_P, _I, _I, ctypes.POINTER(GridDesc), _I, ctypes.POINTER(_Z)])(
                _hval(handle), eb, n, self._descs, self.solvedim, ctypes.byref(size))
        if st != SUCCESS:
            raise PentadError(st, "plan buffer size")
        self.buffer_bytes = max(int(size.value), 256)
        if scratch is None or self.refine:
            self.buffer = torch.empty(self.buffer_bytes + 256, dtype=torch.uint8,
                                      device=self.device)
            off = (-self.buffer.data_ptr()) % 256
            self._buf = self.buffer[off:off + self.buffer_bytes]
        self._plan = _P(None)
        # plan creation writes the job table into the new buffer without
        # waiting for other streams: the allocator may have handed out memory
        # that work queued on this stream still uses, so let that finish
        idle = torch.cuda.current_stream(self.device).synchronize
        if scratch is not None and not self.refine:
            # job table in its own small buffer, scratch shared with other
            # plans that never run at the same time
            tb, sb = plan_sizes(self.grids, self.solvedim, handle)
            if scratch.numel() * scratch.element_size() < sb or scratch.data_ptr() % 256:
                raise ValueError(f"scratch needs {sb} bytes, 256-byte aligned")
            self.scratch = scratch
            self.buffer = torch.empty(tb + 512, dtype=torch.uint8, device=self.device)
            off = (-self.buffer.data_ptr()) % 256
            self._buf = self.buffer[off:off + max(tb, 256)]
            idle()
            st = _typed("pentadsolver_plan_create_split",
                        [_P, _I, _I, ctypes.POINTER(GridDesc), _I, _P, _Z, _P, _Z, _I,
                         ctypes.POINTER(_P)])(
                _hval(handle), eb, n, self._descs, self.solvedim, _ptr(self._buf), tb,
                _ptr(scratch), scratch.numel() * scratch.element_size(), int(ctas),
                ctypes.byref(self._plan))
            if st != SUCCESS:
                raise PentadError(st, "plan create")
            return
        idle()
        if self.refine:
            st = _typed("pentadsolver_refine_plan_create",
                        [_P, _I, ctypes.POINTER(GridDesc), _I, _I, _P, _Z, _I, ctypes.POINTER(_P)])(
                _hval(handle), n, self._descs, self.solvedim, int(refine_steps), _ptr(self._buf),
                self.buffer_bytes, int(ctas), ctypes.byref(self._plan))
        else:
            st = _typed("pentadsolver_plan_create",
                        [_P, _I, _I, ctypes.POINTER(GridDesc), _I, _P, _Z, _I, ctypes.POINTER(_P)])(
                _hval(handle), eb, n, self._descs, self.solvedim, _ptr(self._buf),
                self.buffer_bytes, int(ctas), ctypes.byref(self._plan))
        if st != SUCCESS:
            raise PentadError(st, "plan create")

    def execute(self, stream=None, reuse_fp32: bool = False) -> None:
        """Run the plan.  ``reuse_fp32`` (refinement plans): keep the FP32
        coefficient copies of an earlier execute -- the caller vouches that
        the coefficients have not changed (``PENTADSOLVER_PLAN_REUSE_FP32``)."""
        st = _typed("pentadsolver_plan_execute_ex", [_P, _P, _I])(
            self._plan, _stream_ptr(stream, self.device), 1 if reuse_fp32 else 0)
        if st != SUCCESS:
            raise PentadError(st, "plan execute")

    def describe(self) -> str:
        return _typed("pentadsolver_plan_describe", [_P], ctypes.c_char_p)(self._plan).decode()

    def autotune(self, reps: int = 5, stream=None) -> int:
        """Time executes at several CTA counts, keep the fastest for this plan
        and record it in the library's tuning table; returns the CTA count."""
        best = ctypes.c_int(0)
        st = _typed("pentadsolver_autotune_plan", [_P, _I, _P, ctypes.POINTER(_I)])(
            self._plan, int(reps), _stream_ptr(stream, self.device), ctypes.byref(best))
        if st != SUCCESS:
            raise PentadError(st, "plan autotune")
        return int(best.value)

    def status_check(self, stream=None) -> tuple[int, int]:
        """Read and clear this plan's own status bits, then synchronise."""
        bits = ctypes.c_int(0)
        st = _typed("pentadsolver_plan_status_check", [_P, _P, ctypes.POINTER(_I)])(
            self._plan, _stream_ptr(stream, self.device), ctypes.byref(bits))
        return int(st), int(bits.value)

    def estimates(self, stream=None):
        """(max|last correction|, max|x|) per grid of a refinement plan."""
        out = (ctypes.c_double * (2 * len(self.grids)))()
        st = _typed("pentadsolver_plan_estimates", [_P, _P, _P])(
            self._plan, _stream_ptr(stream, self.device), out)
        if st != SUCCESS:
            raise PentadError(st, "plan estimates")
        return [(out[2 * i], out[2 * i + 1]) for i in range(len(self.grids))]

    def close(self) -> None:
        if getattr(self, "_plan", None) and self._plan.value:
            _typed("pentadsolver_plan_destroy", [_P])(self._plan)
            self._plan = _P(None)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refine_buffer_size(dims, solvedim: int, handle=None) -> int:
    size = ctypes.c_size_t(0)
    st = _typed("pentadsolver_refine_buffer_size", [_P, _P, _I, _I, ctypes.POINTER(_Z)])(
        _hval(handle), _dims(dims), len(dims), int(solvedim), ctypes.byref(size))
    if st != SUCCESS:
        raise PentadError(st, "refine buffer size")
    return int(size.value)


def alloc_refine_buffer(dims, solvedim: int, device="cuda"):
    """A 256-byte aligned uint8 view of refine_buffer_size bytes."""
    import torch

    n = refine_buffer_size(dims, solvedim)
    raw = torch.empty(n + 256, dtype=torch.uint8, device=device)
    off = (-raw.data_ptr()) % 256
    return raw[off:off + n]


def gpsv_batch_refine(ds, dl, d, du, dw, x, solvedim: int, steps: int = 1, buffer=None,
                      reuse_fp32_coefficients: bool = False, stream=None, handle=None,
                      check: bool = True) -> int:
    """FP64 solve in place with FP32 sweeps and ``steps`` rounds of FP64
    residual/correction (``pentadsolver_D_gpsv_batch_refine``)."""
    _check_arrays((ds, dl, d, du, dw, x))
    dims = dims_of(x)
    if buffer is None:
        buffer = alloc_refine_buffer(dims, solvedim, x.device)
    st = _typed("pentadsolver_D_gpsv_batch_refine", [_P] * 7 + [_P, _I, _I, _I, _I, _P, _Z, _P])(
        _hval(handle), *(_ptr(a) for a in (ds, dl, d, du, dw, x)), _dims(dims), len(dims),
        int(solvedim), int(steps), int(bool(reuse_fp32_coefficients)), _ptr(buffer),
        buffer.numel() * buffer.element_size(), _stream_ptr(stream, x.device))
    if check and st != SUCCESS:
        raise PentadError(st, "gpsv_batch_refine")
    return st


def refine_estimate(buffer, stream=None) -> tuple[float, float]:
    out = (ctypes.c_double * 2)()
    st = _typed("pentadsolver_refine_estimate", [_P, _P, _P])(
        _ptr(buffer), _stream_ptr(stream, buffer.device), out)
    if st != SUCCESS:
        raise PentadError(st, "refine estimate")
    return out[0], out[1]


def set_tuning(handle, direction: int, spec: str | None) -> None:
    """pentadsolver_set_tuning: "auto", "no-tmem", "no-tma", "tmem=ST,XST",
    "tma=R,ST,XST,SCR" for one direction of a handle."""
    st = _typed("pentadsolver_set_tuning", [_P, _I, ctypes.c_char_p])(
        _hval(handle), int(direction), None if spec is None else spec.encode())
    if st != SUCCESS:
        raise PentadError(st, f"set_tuning({spec!r})")


def plan_sizes(grids, solvedim: int, handle=None) -> tuple[int, int]:
    """(job table bytes, scratch bytes) of a plan over these grids."""
    descs = _grid_descs(grids)
    tb, sb = ctypes.c_size_t(0), ctypes.c_size_t(0)
    st = _typed("pentadsolver_plan_sizes",
                [_P, _I, _I, ctypes.POINTER(GridDesc), _I, ctypes.POINTER(_Z), ctypes.POINTER(_Z)])(
        _hval(handle), grids[0]["x"].element_size(), len(grids), descs, int(solvedim),
        ctypes.byref(tb), ctypes.byref(sb))
    if st != SUCCESS:
        raise PentadError(st, "plan sizes")
    return int(tb.value), int(sb.value)


def aligned_bytes(n: int, device="cuda"):
    """A 256-byte aligned uint8 view of n bytes."""
    import torch

    raw = torch.empty(n + 256, dtype=torch.uint8, device=device)
    off = (-raw.data_ptr()) % 256
    return raw[off:off + n]


# ---------------------------------------------------------------------------
# The library's tuning table and autotuner
# ---------------------------------------------------------------------------
def tuning_load(path) -> None:
    st = _typed("pentadsolver_tuning_load", [ctypes.c_char_p])(os.fsencode(str(path)))
    if st != SUCCESS:
        raise PentadError(st, f"tuning_load {path}")


def tuning_save(path) -> None:
    st = _typed("pentadsolver_tuning_save", [ctypes.c_char_p])(os.fsencode(str(path)))
    if st != SUCCESS:
        raise PentadError(st, f"tuning_save {path}")


def tuning_clear() -> None:
    _typed("pentadsolver_tuning_clear", [])()


def tuning_set(key: str, spec: str = "auto", algo: str = "auto", lanes: int = 0, ctas: int = 0,
               ms: float = 0.0) -> None:
    st = _typed("pentadsolver_tuning_set",
                [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, _I, _I, ctypes.c_double])(
        key.encode(), spec.encode(), algo.encode(), int(lanes), int(ctas), float(ms))
    if st != SUCCESS:
        raise PentadError(st, "tuning_set")


def tuning_lookup(key: str) -> dict | None:
    """The table's entry for ``key`` (spec, algo, lanes, ctas, ms), or None."""
    out = ctypes.create_string_buffer(512)
    st = _typed("pentadsolver_tuning_lookup", [ctypes.c_char_p, ctypes.c_char_p, _Z])(
        key.encode(), out, 512)
    if st != SUCCESS:
        return None
    spec, algo, lanes, ctas, ms = out.value.decode().split("\t")
    return {"spec": spec, "algo": algo, "lanes": int(lanes), "ctas": int(ctas), "ms": float(ms)}


def tuning_key(dims, solvedim: int, elem_bytes: int = 8, kind: str = "solve",
               gpu_name: str | None = None) -> str:
    out = ctypes.create_string_buffer(512)
    st = _typed("pentadsolver_tuning_key",
                [ctypes.c_char_p, ctypes.c_char_p, _I, _P, _I, _I, ctypes.c_char_p, _Z])(
        None if gpu_name is None else gpu_name.encode(), kind.encode(), int(elem_bytes),
        _dims(dims), len(dims), int(solvedim), out, 512)
    if st != SUCCESS:
        raise PentadError(st, "tuning_key")
    return out.value.decode()


def autotune_solve(ds, dl, d, du, dw, x, solvedim: int, reps: int = 5, buffer=None,
                   x_save=None, stream=None, handle=None) -> list[dict]:
    """The library's autotuner on this problem: every distinct candidate's
    time, fastest first (the first is now in the tuning table)."""
    _check_arrays((ds, dl, d, du, dw, x))
    pre, eb = _elem_prefix(x.dtype)
    dims = dims_of(x)
    if buffer is None:
        buffer = alloc_buffer(dims, solvedim, x.dtype, x.device)
    nbytes = buffer.numel() * buffer.element_size()
    out = ctypes.create_string_buffer(8192)
    st = _typed("pentadsolver_autotune_solve",
                [_P, _I] + [_P] * 7 + [_P, _I, _I, _P, _Z, _I, _P, ctypes.c_char_p, _Z])(
        _hval(handle), eb, *(_ptr(a) for a in (ds, dl, d, du, dw, x)),
        None if x_save is None else _ptr(x_save), _dims(dims), len(dims), int(solvedim),
        _ptr(buffer), nbytes, int(reps), _stream_ptr(stream, x.device), out, 8192)
    if st != SUCCESS:
        raise PentadError(st, "autotune_solve")
    rows = []
    for line in out.value.decode().splitlines():
        label, spec, algo, lanes, variant, ms = line.split("\t")
        rows.append({"label": label, "spec": spec, "algo": algo, "lanes": int(lanes),
                     "variant": variant, "ms": float(ms)})
    return rows


# ---------------------------------------------------------------------------
# Slab decomposition (the data movement around the all-to-all)
# ---------------------------------------------------------------------------
def _slab_call(name, elem_bytes, src, dst, nx, ny, nz_local, parts, stream):
    sp = None
    if stream is not None:
        sp = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
    return int(_typed(name, [_I, _P, _P, _I, _I, _I, _I, _P])(
        int(elem_bytes), _ptr(src), _ptr(dst), int(nx), int(ny), int(nz_local), int(parts), sp))


def slab_pack(elem_bytes, zslab, send, nx, ny, nz_local, parts, stream=None) -> int:
    """send[r][zl][yl][x] = zslab[zl][r ny/parts + yl][x] (pentadsolver_slab_pack)."""
    return _slab_call("pentadsolver_slab_pack", elem_bytes, zslab, send, nx, ny, nz_local,
                      parts, stream)


def slab_unpack(elem_bytes, recv, zslab, nx, ny, nz_local, parts, stream=None) -> int:
    """zslab[zl][r ny/parts + yl][x] = recv[r][zl][yl][x] (pentadsolver_slab_unpack)."""
    return _slab_call("pentadsolver_slab_unpack", elem_bytes, recv, zslab, nx, ny, nz_local,
                      parts, stream)
