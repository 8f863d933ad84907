"""ADI iterations captured once and replayed as one CUDA graph.

An ADI time step solves the same grid in place along x, then y, then z, with
coefficient arrays that do not change between steps -- the loop of the
reference's application (apps/adi_cuda.cu:167-176), which makes one
``pentadsolver_gpsv_batch`` call per direction.  ``AdiGraph`` records
``iterations`` such steps (3 x iterations solves through the library's C ABI)
into one CUDA graph; a replay launches them all with one call and none of the
host work between launches.  With shared factorisation the factor tables stay
cached in the buffer across all steps, so the serial recurrences run once.

Everything host-side that a solve sets up once (occupancy queries, the
tensor-map encoder, kernel attributes) is done by a warm-up pass on a copy of
the right-hand side before capture, so ``x`` is untouched until the first
replay.
"""
from __future__ import annotations

import pentadsolver as ps


class AdiGraph:
    def __init__(self, ds, dl, d, du, dw, x, iterations: int = 1, algo: str | None = None,
                 buffer=None, handle=None):
        import torch

        self.arrays = (ds, dl, d, du, dw, x)
        self.iterations = int(iterations)
        self.ndim = x.dim()
        self._own_handle = handle is None
        self.handle = ps.Handle() if handle is None else handle
        if algo is not None:
            for direction in range(self.ndim):
                self.handle.set_algo(direction, algo)
        dims = ps.dims_of(x)
        # the x direction needs the largest buffer (the reference's sizing)
        self.buffer = buffer if buffer is not None else ps.alloc_buffer(dims, 0, x.dtype,
                                                                         x.device)
        self.stream = torch.cuda.Stream(device=x.device)
        # warm-up on a copy: one solve per direction
        scratch = x.clone()
        with torch.cuda.stream(self.stream):
            for axis in range(self.ndim):
                ps.gpsv_batch(ds, dl, d, du, dw, scratch, axis, buffer=self.buffer,
                              stream=self.stream, handle=self.handle)
        self.stream.synchronize()
        del scratch
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            for _ in range(self.iterations):
                for axis in range(self.ndim):
                    ps.gpsv_batch(ds, dl, d, du, dw, x, axis, buffer=self.buffer,
                                  stream=self.stream, handle=self.handle)

    @property
    def launches(self) -> int:
        """Solves (kernel launches of the library) per replay."""
        return self.iterations * self.ndim

    def replay(self) -> None:
        """Run the captured steps on x in place (on the current stream's order)."""
        self.graph.replay()

    def kernels(self) -> list[str]:
        """The kernel family each direction ran (``pentadsolver_kernel_that_ran``)."""
        return [self.handle.kernel_that_ran(a) for a in range(self.ndim)]

    def close(self) -> None:
        self.graph = None
        if self._own_handle and self.handle is not None:
            self.handle.close()
        self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
