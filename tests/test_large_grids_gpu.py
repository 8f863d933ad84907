"""Grids of 2^31 points and more on the Tensor-Memory kernel.

An FP32 grid of 1024 x 1024 x 2049 points (2.15e9, 8.6 GB per array) is
solved along x and along y.  Lines are independent, so the first and the last
lines of the grid -- the last ones beyond element offset 2^31, where any
32-bit offset would wrap -- solved as grids of their own must give the same
bits as in the full solve (the same tiles of 16 lines, the same arithmetic),
and they must match the oracle.  About 100 GB of device memory.
"""
import numpy as np
import pytest

import pentadsolver as ps
from gpu_util import fwd_err
from oracle import oracle

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

DIMS = (1024, 1024, 2049)
NAMES = ("ds", "dl", "d", "du", "dw")


@pytest.fixture(scope="module")
def big(cuda):
    import torch

    if torch.cuda.get_device_properties(0).total_memory < 150e9:
        pytest.skip("needs a device with ~100 GB free")
    g = torch.Generator(device="cuda").manual_seed(2031)
    n = int(np.prod(DIMS))
    assert n >= 1 << 31

    def u(lo, hi):
        t = torch.rand(n, generator=g, device="cuda", dtype=torch.float32)
        return t.mul_(hi - lo).add_(lo)

    co = {k: u(-1, 1) for k in ("ds", "dl", "du", "dw")}
    d = u(1, 2)
    for k in ("ds", "dl", "du", "dw"):
        d.add_(co[k].abs())
    co["d"] = d
    co["b"] = u(-1, 1)
    yield co
    co.clear()
    torch.cuda.empty_cache()


def _solve(co, x, dims, solvedim, h):
    import torch

    need = 3 * int(np.prod(dims)) * 4 + 256   # any scratch the kernel may take
    buf = torch.empty(need, dtype=torch.uint8, device="cuda")
    ps.gpsv_batch(*(co[k] for k in NAMES), x, solvedim, buffer=buf, dims=dims, handle=h)
    torch.cuda.synchronize()
    del buf


def _sub(co, start, count):
    return {k: co[k][start:start + count] for k in NAMES}


@pytest.mark.parametrize("solvedim", [0, 1])
def test_lines_past_offset_2_31_solve_exactly(big, solvedim):
    import torch

    nx, ny, nz = DIMS
    # the lines compared: along x, 64 whole rows at each end; along y, the
    # first and the last z plane (1024 runs of 1024 lines each)
    if solvedim == 0:
        span, sub_dims = 64 * nx, [nx, 64, 1]
    else:
        span, sub_dims = nx * ny, [nx, ny, 1]
    total = int(np.prod(DIMS))
    heads = [(0, big["b"][:span].clone()), (total - span, big["b"][total - span:].clone())]
    assert heads[1][0] >= 1 << 31
    x = big["b"].clone()
    with ps.Handle() as h:
        _solve(big, x, list(DIMS), solvedim, h)
        d = 0 if solvedim == 0 else 1
        assert "tmem" in h.variant_that_ran(d), h.variant_that_ran(d)
        assert ps.status_check(handle=h) == (ps.SUCCESS, 0)
        for start, rhs in heads:
            part = _sub(big, start, span)
            xs = rhs.clone()
            _solve(part, xs, sub_dims, solvedim, h)
            assert torch.equal(xs.view(torch.int32), x[start:start + span].view(torch.int32)), start
            host = {k: v.cpu().numpy() for k, v in part.items()}
            xr = rhs.cpu().numpy().copy()
            oracle.solve(host["ds"], host["dl"], host["d"], host["du"], host["dw"], xr,
                         solvedim, dims=sub_dims)
            assert fwd_err(xs.cpu().numpy(), xr) <= 1e-5, start
    del x
    torch.cuda.empty_cache()
