"""GPU: the random benchmark mesh generated on the device, and fixtures
uploaded and solved.

* ``pentadsolver_{D,S}_mesh_random`` writes, bit for bit, the grid the
  reference's ``Mesh<Float>(solve_dim, dims)`` builds with the same number of
  OpenMP threads (``include/util/mesh.hpp:85-124``) -- checked against the
  oracle restatement, which the CPU tests pin to the reference itself --
  for ragged shapes, every solve dimension, thread counts from 1 to more
  threads than systems, and a 96^3 grid.
* A fixture read by the library and uploaded (the ``DeviceMesh(file)`` path of
  ``test/cuda/singlenode/cuda_tests.cu:8-39``) solves to the fixture's stored
  solution within the reference test's tolerance.
"""
import numpy as np
import pytest

import fixtures
import mesh
import pentadsolver as ps
from gpu_util import NAMES, allclose_ref
from oracle import oracle

pytestmark = pytest.mark.gpu

CASES = [((5,), 0), ((9, 7), 1), ((16, 9, 5), 0), ((16, 9, 5), 1), ((16, 9, 5), 2),
         ((33, 17, 4), 1), ((1, 4, 3), 0), ((2, 5, 3), 0), ((1, 1, 1), 2), ((40, 3, 30), 2),
         ((257, 3, 2), 0)]


def same_bits(a, b):
    return np.array_equal(np.ascontiguousarray(a).view(np.uint8),
                          np.ascontiguousarray(b).view(np.uint8))


@pytest.mark.parametrize("dims,solvedim", CASES)
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_device_mesh_is_the_reference_mesh(cuda, dims, solvedim, dtype):
    import torch

    tdt, ndt = (torch.float64, np.float64) if dtype == "f64" else (torch.float32, np.float32)
    for threads in (1, 3, 8, 64, 700):
        got = mesh.random_mesh(dims, solvedim, threads, tdt, cuda)
        want = oracle.mesh_random(dims, solvedim, threads, ndt)
        torch.cuda.synchronize()
        for k in mesh.NAMES:
            assert same_bits(got[k].cpu().numpy(), want[k]), (dims, solvedim, threads, k)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_device_mesh_96cube(cuda, dtype):
    import torch

    tdt, ndt = (torch.float64, np.float64) if dtype == "f64" else (torch.float32, np.float32)
    for solvedim, threads in ((0, 48), (2, 13)):
        got = mesh.random_mesh((96, 96, 96), solvedim, threads, tdt, cuda)
        want = oracle.mesh_random((96, 96, 96), solvedim, threads, ndt)
        torch.cuda.synchronize()
        for k in mesh.NAMES:
            assert same_bits(got[k].cpu().numpy(), want[k]), (solvedim, k)


def test_device_mesh_on_a_side_stream(cuda):
    import torch

    s = torch.cuda.Stream(device=cuda)
    with torch.cuda.stream(s):
        got = mesh.random_mesh((20, 6, 7), 1, 5, torch.float64, cuda, stream=s)
    s.synchronize()
    want = oracle.mesh_random((20, 6, 7), 1, 5, np.float64)
    assert same_bits(got["x"].cpu().numpy(), want["x"])


@pytest.mark.parametrize("fam,solvedim", [("two_dim_small", 0), ("two_dim_small", 1),
                                          ("two_dim_large", 1), ("one_dim_large", 0)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_fixture_file_uploaded_and_solved(cuda, tmp_path, fam, solvedim, dtype):
    import torch

    fx = fixtures.load_fixture(fam, solvedim)
    path = tmp_path / "case.txt"
    # the reference generator's layout and tokens (test/gen_testcases.py:50-79)
    lines = [f"{len(fx['dims'])} {solvedim}", " ".join(str(v) for v in fx["dims"])]
    lines += [" ".join(str(float(v)) for v in fx[k].ravel()) for k in fixtures.NAMES]
    path.write_text("\n".join(lines) + "\n")
    dev = mesh.fixture_to_device(path, dtype, cuda)
    assert dev["dims"] == fx["dims"] and dev["solvedim"] == solvedim
    buf = ps.alloc_buffer(dev["dims"], solvedim, dev["x"].dtype, cuda)
    ps.gpsv_batch(*(dev[k] for k in NAMES), solvedim, buffer=buf)
    torch.cuda.synchronize()
    ok, worst = allclose_ref(dev["x"].cpu().numpy(), dev["u"], dtype)
    assert ok, worst
