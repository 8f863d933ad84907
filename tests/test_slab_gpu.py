"""The slab-decomposed ADI's kernels and pipeline on one GPU.

* pentadsolver_slab_pack / _unpack against the numpy restatement of their
  block map (16-byte vector and element paths, FP64 and FP32).
* Whole ADI iterations of one grid held as 2 and 4 slabs on this GPU
  ("virtual ranks": the all-to-all done as device copies) through the
  library's solves and pack kernels equal the oracle's x, y, z solves of the
  whole grid.  Between processes the same pipeline exchanges with an NCCL
  all-to-all (slab.nccl_exchange); this run has one GPU.
"""
import numpy as np
import pytest

import fixtures
import pentadsolver as ps
import slab
from gpu_util import fwd_err
from oracle import oracle
from test_slab import np_pack, np_unpack

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims,parts", [((16, 8, 6), 2), ((7, 12, 6), 3), ((33, 16, 8), 4),
                                        ((256, 64, 16), 8), ((5, 4, 4), 1)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_pack_and_unpack_match_the_block_map(cuda, dims, parts, dtype):
    import torch

    L = slab.SlabLayout(dims[0], dims[1], dims[2] * parts, parts)
    rng = np.random.default_rng(3)
    a = rng.standard_normal(L.count).astype(dtype)
    src = torch.from_numpy(a).cuda()
    send = torch.empty_like(src)
    eb = np.dtype(dtype).itemsize
    assert ps.slab_pack(eb, src, send, L.nx, L.ny, L.nzl, parts) == ps.SUCCESS
    torch.cuda.synchronize()
    assert np.array_equal(send.cpu().numpy(), np_pack(a, L))
    back = torch.empty_like(src)
    assert ps.slab_unpack(eb, send, back, L.nx, L.ny, L.nzl, parts) == ps.SUCCESS
    torch.cuda.synchronize()
    assert np.array_equal(back.cpu().numpy(), a)
    assert np.array_equal(np_unpack(np_pack(a, L), L), a)


def test_pack_rejects_bad_arguments(cuda):
    import torch

    t = torch.zeros(64, dtype=torch.float64, device="cuda")
    u = torch.zeros(64, dtype=torch.float64, device="cuda")
    assert ps.slab_pack(8, t, u, 4, 3, 4, 2) == ps.INVALID_VALUE   # ny % parts
    assert ps.slab_pack(8, t, t, 4, 4, 4, 2) == ps.INVALID_VALUE   # in place
    assert ps.slab_pack(2, t, u, 4, 4, 4, 2) == ps.INVALID_VALUE   # element size


@pytest.mark.parametrize("dims,parts", [((64, 48, 40), 2), ((33, 20, 24), 4), ((40, 32, 32), 1)])
def test_slab_adi_on_virtual_ranks_equals_the_oracle(cuda, dims, parts):
    import torch

    nx, ny, nz = dims
    L = slab.SlabLayout(nx, ny, nz, parts)
    co = fixtures.random_dominant(dims, 77, np.float64)
    coefs, xs = [], []
    for k in range(parts):
        z0, z1 = L.z_range(k)
        coefs.append({n: torch.from_numpy(np.ascontiguousarray(co[n][z0:z1])).cuda()
                      for n in slab.NAMES})
        xs.append(torch.from_numpy(np.ascontiguousarray(co["x"][z0:z1])).cuda())
    with ps.Handle() as h:
        adi = slab.SlabADI(L, coefs, slab.local_exchange(L), handle=h)
        for _ in range(2):
            adi.iterate(xs)
        torch.cuda.synchronize()
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
    got = torch.cat(xs, 0).cpu().numpy()
    x = co["x"].copy()
    for _ in range(2):
        for axis in range(3):
            oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], x, axis)
    assert fwd_err(got, x) <= 1e-12
