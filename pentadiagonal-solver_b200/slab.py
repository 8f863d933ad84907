"""Slab-decomposed ADI over several GPUs: one grid, one slab per rank.

The reference distributes a solve over MPI ranks with a reduced-system
exchange staged through host memory (``src/cuda/mpi/pentad_cuda.cu:929-955``,
``:529-555``).  Here the ADI iteration of a grid split into slabs along z runs
as

  x solve, y solve      on the rank's z slab (lines inside the slab);
  pack + all-to-all     z slabs -> y slabs (one exchange of equal blocks);
  z solve               on the rank's y slab (z lines now inside it);
  all-to-all + unpack   y slabs -> z slabs.

Every solve is the library's single-GPU solve; the coefficient arrays of the
z solve are transposed once, at set-up, and stay in y-slab layout.  The
exchange is an NCCL all-to-all over NVLink between processes (one rank per
GPU).  A process may also hold several slabs ("virtual ranks"): their
exchange is then the same block transposition done with device copies,
which is how the pipeline is checked on one GPU.

Layout (``SlabLayout``): a global grid nx x ny x nz (x contiguous), `parts`
ranks; rank k's z slab holds z in [k nzl, (k+1) nzl) as [zl][y][x]
(nzl = nz / parts); its y slab holds y in [k nyp, (k+1) nyp), all z, as
[z][yl][x] (nyp = ny / parts).  The pack/unpack kernels and the block
arithmetic are those of ``csrc/slab_kernels.cu``.
"""
from __future__ import annotations

from dataclasses import dataclass

NAMES = ("ds", "dl", "d", "du", "dw")


@dataclass(frozen=True)
class SlabLayout:
    nx: int
    ny: int
    nz: int
    parts: int

    def __post_init__(self):
        if min(self.nx, self.ny, self.nz, self.parts) < 1:
            raise ValueError("extents and parts must be positive")
        if self.ny % self.parts or self.nz % self.parts:
            raise ValueError("ny and nz must be multiples of the number of slabs")

    @property
    def nzl(self) -> int:
        return self.nz // self.parts

    @property
    def nyp(self) -> int:
        return self.ny // self.parts

    @property
    def count(self) -> int:
        """Points per slab (the same in both layouts)."""
        return self.nx * self.ny * self.nzl

    def zslab_dims(self) -> list[int]:
        return [self.nx, self.ny, self.nzl]

    def yslab_dims(self) -> list[int]:
        return [self.nx, self.nyp, self.nz]

    def z_range(self, rank: int) -> tuple[int, int]:
        return rank * self.nzl, (rank + 1) * self.nzl

    def y_range(self, rank: int) -> tuple[int, int]:
        return rank * self.nyp, (rank + 1) * self.nyp


def nccl_exchange(group=None):
    """The all-to-all of equal blocks between processes (one slab each)."""
    import torch.distributed as dist

    def exchange(sends, recvs):
        assert len(sends) == len(recvs) == 1
        dist.all_to_all_single(recvs[0], sends[0], group=group)

    return exchange


def local_exchange(layout: SlabLayout):
    """The same exchange among the slabs one process holds: block r of rank
    k's send buffer becomes block k of rank r's receive buffer."""
    blk = layout.count // layout.parts

    def exchange(sends, recvs):
        assert len(sends) == len(recvs) == layout.parts
        for k, snd in enumerate(sends):
            for r, rcv in enumerate(recvs):
                rcv[k * blk:(k + 1) * blk].copy_(snd[r * blk:(r + 1) * blk])

    return exchange


class SlabADI:
    """ADI iterations of a slab-decomposed grid.

    ``coefficients``: per slab this process holds, a dict of the five
    coefficient arrays in z-slab layout (flat or shaped tensors of
    ``layout.count`` elements); ``ranks``: the global ranks of those slabs.
    ``exchange(sends, recvs)`` performs the all-to-all (``nccl_exchange`` /
    ``local_exchange``).  ``solve`` and ``pack`` default to the library's CUDA
    solve and pack/unpack kernels.
    """

    def __init__(self, layout: SlabLayout, coefficients, exchange, ranks=None, handle=None,
                 stream=None, solve=None, pack=None, unpack=None):
        import torch

        import pentadsolver as ps

        self.ps = ps
        self.layout = layout
        self.coef_z = [{k: c[k].reshape(-1) for k in NAMES} for c in coefficients]
        self.ranks = list(ranks) if ranks is not None else list(range(len(coefficients)))
        self.exchange = exchange
        self.handle = handle
        self.stream = stream
        self._solve = solve or self._library_solve
        self._pack = pack or self._library_pack
        self._unpack = unpack or self._library_unpack
        ref = self.coef_z[0]["d"]
        self.dtype, self.device = ref.dtype, ref.device
        if self.stream is None and self.device.type == "cuda":
            # solves, pack kernels and the local exchange's copies on one stream
            self.stream = torch.cuda.current_stream(self.device)
        n = layout.count
        self.send = [torch.empty(n, dtype=self.dtype, device=self.device) for _ in self.ranks]
        self.xy = [torch.empty(n, dtype=self.dtype, device=self.device) for _ in self.ranks]
        self.back = [torch.empty(n, dtype=self.dtype, device=self.device) for _ in self.ranks]
        # the z solve's coefficients, transposed once into y-slab layout
        self.coef_y = [{} for _ in self.ranks]
        for k in NAMES:
            for i, c in enumerate(self.coef_z):
                self._pack(c[k], self.send[i])
            recv = [torch.empty(n, dtype=self.dtype, device=self.device) for _ in self.ranks]
            self.exchange(self.send, recv)
            for i in range(len(self.ranks)):
                self.coef_y[i][k] = recv[i]
        self.buffers = {}

    # -- the library's kernels -----------------------------------------------------
    def _buffer(self, dims, solvedim):
        key = (tuple(dims), solvedim)
        if key not in self.buffers:
            self.buffers[key] = self.ps.alloc_buffer(list(dims), solvedim, self.dtype,
                                                     self.device)
        return self.buffers[key]

    def _library_solve(self, coef, x, dims, solvedim):
        self.ps.gpsv_batch(*(coef[k] for k in NAMES), x, solvedim, dims=dims,
                           buffer=self._buffer(dims, solvedim), stream=self.stream,
                           handle=self.handle)

    def _elem(self):
        return 8 if self.dtype.itemsize == 8 else 4

    def _library_pack(self, src, dst):
        L = self.layout
        st = self.ps.slab_pack(self._elem(), src, dst, L.nx, L.ny, L.nzl, L.parts, self.stream)
        if st != self.ps.SUCCESS:
            raise self.ps.PentadError(st, "slab pack")

    def _library_unpack(self, src, dst):
        L = self.layout
        st = self.ps.slab_unpack(self._elem(), src, dst, L.nx, L.ny, L.nzl, L.parts,
                                 self.stream)
        if st != self.ps.SUCCESS:
            raise self.ps.PentadError(st, "slab unpack")

    # -- one ADI iteration ---------------------------------------------------------
    def iterate(self, xs) -> None:
        """x, then y, then z on every slab held here; `xs` (z-slab layout,
        one tensor per slab) are solved in place."""
        L = self.layout
        zd, yd = L.zslab_dims(), L.yslab_dims()
        flat = [x.reshape(-1) for x in xs]
        for c, x in zip(self.coef_z, flat):
            self._solve(c, x, zd, 0)
            self._solve(c, x, zd, 1)
        for i, x in enumerate(flat):
            self._pack(x, self.send[i])
        self.exchange(self.send, self.xy)
        for c, xy in zip(self.coef_y, self.xy):
            self._solve(c, xy, yd, 2)
        self.exchange(self.xy, self.back)
        for i, x in enumerate(flat):
            self._unpack(self.back[i], x)
