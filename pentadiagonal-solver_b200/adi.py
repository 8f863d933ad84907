"""ADI iterations captured once and replayed as one CUDA graph.

An ADI time step solves the same grid in place along x, then y, then z, with
coefficient arrays that do not change between steps -- the loop of the
reference's application (apps/adi_cuda.cu:167-176), which makes one
``pentadsolver_gpsv_batch`` call per direction.  ``AdiGraph`` is the Python
front end of the library's ``pentadsolver_adi_create``: ``iterations`` such
steps (3 x iterations solves through the library's C ABI) recorded into one
CUDA graph; a replay launches them all with one call and none of the host
work between launches.  With shared factorisation the factor tables stay
cached in the buffer across all steps, so the serial recurrences run once.
The library warms up (kernel attributes, occupancy queries, tensor maps) on a
copy of x kept in the buffer's unused tail, so x is untouched until the
first replay.
"""
from __future__ import annotations

import ctypes

import pentadsolver as ps


class AdiGraph:
    def __init__(self, ds, dl, d, du, dw, x, iterations: int = 1, algo: str | None = None,
                 buffer=None, handle=None):
        self.arrays = (ds, dl, d, du, dw, x)
        self.iterations = int(iterations)
        self.ndim = x.dim()
        self.device = x.device
        self._own_handle = handle is None
        self.handle = ps.Handle() if handle is None else handle
        if algo is not None:
            for direction in range(self.ndim):
                self.handle.set_algo(direction, algo)
        dims = ps.dims_of(x)
        # the x direction's reference-sized buffer (the largest)
        self.buffer = buffer if buffer is not None else ps.alloc_buffer(dims, 0, x.dtype,
                                                                         x.device)
        _, eb = ps._elem_prefix(x.dtype)
        self._adi = ctypes.c_void_p(None)
        st = ps._typed("pentadsolver_adi_create",
                       [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_void_p] * 7 +
                       [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t,
                        ctypes.POINTER(ctypes.c_void_p)])(
            ps._hval(self.handle), eb, *(ps._ptr(a) for a in self.arrays), ps._dims(dims),
            len(dims), self.iterations, ps._ptr(self.buffer),
            self.buffer.numel() * self.buffer.element_size(), ctypes.byref(self._adi))
        if st != ps.SUCCESS:
            raise ps.PentadError(st, "adi graph create")

    @property
    def launches(self) -> int:
        """Solves (kernel launches of the library) per replay."""
        return int(ps._typed("pentadsolver_adi_launches", [ctypes.c_void_p])(self._adi))

    def replay(self, stream=None) -> None:
        """Run the captured steps on x in place, on `stream` (default: the
        current stream)."""
        st = ps._typed("pentadsolver_adi_replay", [ctypes.c_void_p, ctypes.c_void_p])(
            self._adi, ps._stream_ptr(stream, self.device))
        if st != ps.SUCCESS:
            raise ps.PentadError(st, "adi graph replay")

    def kernels(self) -> list[str]:
        """The kernel family each direction ran (``pentadsolver_kernel_that_ran``)."""
        return [self.handle.kernel_that_ran(a) for a in range(self.ndim)]

    def close(self) -> None:
        if getattr(self, "_adi", None) is not None and self._adi.value:
            ps._typed("pentadsolver_adi_destroy", [ctypes.c_void_p])(self._adi)
            self._adi = ctypes.c_void_p(None)
        if self._own_handle and getattr(self, "handle", None) is not None:
            self.handle.close()
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
