"""The slab-decomposed ADI's host logic on CPU.

* Layout arithmetic and its limits.
* The pack / exchange / unpack block transposition (here with a numpy
  restatement of the pack map; the CUDA kernels are checked against the same
  map in test_slab_gpu.py) turns z slabs into y slabs and back.
* Two gloo ranks on 127.0.0.1 run whole ADI iterations of one grid split in
  two slabs -- x and y solved in the z slabs, an all-to-all, z solved in the
  y slabs, an all-to-all back -- with the oracle as the per-slab solver, and
  the gathered result equals the oracle's x, y, z solves of the whole grid.
"""
import datetime
import json
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

import fixtures
import slab

REPO = Path(__file__).resolve().parents[1]


def np_pack(a, layout):
    """send[r][zl][yl][x] = zslab[zl][r nyp + yl][x] (the kernels' map)."""
    L = layout
    return np.ascontiguousarray(
        a.reshape(L.nzl, L.parts, L.nyp, L.nx).transpose(1, 0, 2, 3)).reshape(-1)


def np_unpack(p, layout):
    L = layout
    return np.ascontiguousarray(
        p.reshape(L.parts, L.nzl, L.nyp, L.nx).transpose(1, 0, 2, 3)).reshape(-1)


def test_layout():
    L = slab.SlabLayout(12, 8, 6, 2)
    assert (L.nzl, L.nyp, L.count) == (3, 4, 12 * 8 * 3)
    assert L.zslab_dims() == [12, 8, 3] and L.yslab_dims() == [12, 4, 6]
    assert L.z_range(1) == (3, 6) and L.y_range(1) == (4, 8)
    for bad in ((12, 7, 6, 2), (12, 8, 5, 2), (12, 8, 6, 0)):
        with pytest.raises(ValueError):
            slab.SlabLayout(*bad)


@pytest.mark.parametrize("parts", [1, 2, 4])
def test_block_transposition_gives_y_slabs_and_back(parts):
    import torch

    nx, ny, nz = 5, 8, 12
    L = slab.SlabLayout(nx, ny, nz, parts)
    grid = np.arange(nx * ny * nz, dtype=np.float64).reshape(nz, ny, nx)
    zs = [grid[slice(*L.z_range(k))] for k in range(parts)]
    sends = [torch.from_numpy(np_pack(z, L)) for z in zs]
    recvs = [torch.empty(L.count, dtype=torch.float64) for _ in range(parts)]
    slab.local_exchange(L)(sends, recvs)
    for r in range(parts):   # rank r holds y in its range, all z, as [z][yl][x]
        want = grid[:, slice(*L.y_range(r)), :]
        assert np.array_equal(recvs[r].numpy().reshape(nz, L.nyp, nx), want)
    back = [torch.empty(L.count, dtype=torch.float64) for _ in range(parts)]
    slab.local_exchange(L)(recvs, back)
    for k in range(parts):
        assert np.array_equal(np_unpack(back[k].numpy(), L).reshape(L.nzl, ny, nx), zs[k])


def _cpu_hooks(layout):
    from oracle import oracle

    def solve(coef, x, dims, solvedim):
        c = {k: coef[k].numpy() for k in slab.NAMES}
        oracle.solve(c["ds"], c["dl"], c["d"], c["du"], c["dw"], x.numpy(), solvedim, dims=dims)

    def pack(src, dst):
        dst.copy_(__import__("torch").from_numpy(np_pack(src.numpy(), layout)))

    def unpack(src, dst):
        dst.copy_(__import__("torch").from_numpy(np_unpack(src.numpy(), layout)))

    return solve, pack, unpack


DIMS = (10, 8, 12)   # nx, ny, nz


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    L = slab.SlabLayout(*DIMS, world)
    co = fixtures.random_dominant(DIMS, 2024, np.float64)
    z0, z1 = L.z_range(rank)
    mine = {k: torch.from_numpy(np.ascontiguousarray(co[k][z0:z1])) for k in co}
    solve, pack, unpack = _cpu_hooks(L)
    adi = slab.SlabADI(L, [mine], slab.nccl_exchange(), ranks=[rank], solve=solve, pack=pack,
                       unpack=unpack)
    x = mine["x"].clone()
    for _ in range(2):
        adi.iterate([x])
    parts = [torch.empty_like(x) for _ in range(world)]
    dist.all_gather(parts, x)
    dist.barrier()
    dist.destroy_process_group()
    if rank == 0:
        np.save(Path(out_dir) / "x.npy", torch.cat(parts, 0).numpy())


def test_two_gloo_ranks_run_the_slab_adi(tmp_path):
    import torch.multiprocessing as mp

    from oracle import oracle

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(tmp_path / "x.npy")
    co = fixtures.random_dominant(DIMS, 2024, np.float64)
    x = co["x"].copy()
    for _ in range(2):
        for axis in range(3):
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x, axis)
    assert got.shape == x.shape
    assert float(np.abs(got - x).max() / np.abs(x).max()) <= 1e-12
