"""GPU: the reference's own programs and GPU solver against this library.

* The reference's verification apps (``apps/verify_strided_cuda.cu``,
  ``verify_shared_fact_cuda.cu``, ``verify_scale_cuda.cu``,
  ``fp32_accuracy_cuda.cu``), unchanged and built by ``oracle/Makefile`` on this
  library, pass their own checks: full-grid backward residuals and cross-kernel
  differences at the reference's tolerances (1e-10 FP64, 1e-3 FP32 strided;
  shared factorisation against the general path), and the FP32 forward error
  against their host FP64 Thomas reference.
* The reference's ADI benchmark app runs on this library and reports the
  kernels it expects.
* Plain FP64 results equal the reference's own CUDA solver
  (``src/cuda/singlenode/pentad_cuda.cu``, compiled into ``oracle/_ref``) within
  1e-12 forward error on the same device arrays, every solve dimension.
"""
import ctypes
import os
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import fixtures
import pentadsolver as ps
from gpu_util import NAMES, fwd_err, to_dev
from oracle import oracle

pytestmark = pytest.mark.gpu

REF = Path(__file__).resolve().parent.parent / "oracle" / "_ref"


def run_app(name, *args, env=None, timeout=600):
    exe = REF / name
    if not exe.exists():
        pytest.skip(f"{exe} not built (oracle/Makefile ref)")
    e = {k: v for k, v in os.environ.items() if not k.startswith("PENTA_")}
    e.update(env or {})
    r = subprocess.run([str(exe), *map(str, args)], env=e, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    assert "CUDA error" not in r.stderr, r.stderr[-2000:]
    return r.stdout


@pytest.mark.parametrize("prec", ["double", "float"])
@pytest.mark.parametrize("direction", [1, 2])
def test_reference_verify_strided(cuda, prec, direction):
    out = run_app("verify_strided_cuda_b200", 256, prec, direction, "thomas-pcr")
    assert "PASS" in out and "FAIL" not in out, out


@pytest.mark.parametrize("prec", ["double", "float"])
@pytest.mark.parametrize("solvedim", [0, 1, 2])
def test_reference_verify_shared_fact(cuda, prec, solvedim):
    out = run_app("verify_shared_fact_cuda_b200", 256, prec, solvedim)
    assert "PASS" in out and "FAIL" not in out, out


@pytest.mark.parametrize("n,prec", [(256, "double"), (255, "double"), (100, "float"),
                                    (512, "double")])
def test_reference_verify_scale(cuda, n, prec):
    out = run_app("verify_scale_cuda_b200", n, prec)
    assert "PASS" in out and "FAIL" not in out, out


@pytest.mark.parametrize("prec,algo,bound", [("float", None, 1e-5), ("double", None, 1e-12),
                                             ("float", "thomas-pcr", 1e-5),
                                             ("float", "naive", 1e-5)])
def test_reference_fp32_accuracy(cuda, prec, algo, bound):
    env = {"PENTA_XALGO": algo} if algo else None
    out = run_app("fp32_accuracy_cuda_b200", 256, prec, 2048, env=env)
    m = re.search(r"forward : max\|x_gpu - x_ref\| = \S+\s+\(rel to max\|x_ref\|=\S+ -> (\S+)\)",
                  out)
    assert m, out
    assert float(m.group(1)) <= bound, out


def test_reference_adi_app_runs_on_this_library(cuda):
    out = run_app("app_cuda_b200", 64, 5, "double")
    csv = [ln for ln in out.splitlines() if ln.startswith("CSV,")]
    assert csv, out
    f = csv[-1].split(",")
    assert [f[2], f[4], f[6]] == ["thomas-pcr"] * 3, f
    out = run_app("app_cuda_b200", 64, 5, "double",
                  env={"PENTA_XALGO": "shared-fact", "PENTA_YZALGO": "shared-fact"})
    f = [ln for ln in out.splitlines() if ln.startswith("CSV,")][-1].split(",")
    assert [f[2], f[4], f[6]] == ["shared-fact"] * 3, f


def reference_cuda():
    so = REF / "libpentad_cuda_ref.so"
    if not so.exists():
        pytest.skip(f"{so} not built (oracle/Makefile ref)")
    lib = ctypes.CDLL(str(so))
    f = lib.pentadsolver_D_gpsv_batch
    f.argtypes = [ctypes.c_void_p] * 7 + [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p]
    f.restype = None
    return f


@pytest.mark.parametrize("dims", [(64, 64, 64), (128, 96, 80), (100, 60, 36)])
def test_fp64_equals_reference_cuda(cuda, dims, monkeypatch):
    import torch

    for k in [k for k in os.environ if k.startswith("PENTA_")]:
        monkeypatch.delenv(k)
    ref_solve = reference_cuda()
    co = fixtures.random_dominant(dims, 4242, np.float64)
    for solvedim in range(3):
        dv_ref = to_dev(co)
        buf = ps.alloc_buffer(list(dims), solvedim, torch.float64, cuda)
        cdims = (ctypes.c_int * 3)(*dims)
        torch.cuda.synchronize()
        ref_solve(None, *(int(dv_ref[k].data_ptr()) for k in NAMES), cdims, 3, solvedim,
                  int(buf.data_ptr()))
        torch.cuda.synchronize()
        dv = to_dev(co)
        ps.gpsv_batch(*(dv[k] for k in NAMES), solvedim, buffer=buf)
        torch.cuda.synchronize()
        mine, theirs = dv["x"].cpu().numpy(), dv_ref["x"].cpu().numpy()
        assert fwd_err(mine, theirs) <= 1e-12, (dims, solvedim)
        want = co["x"].copy()
        oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], want, solvedim)
        assert fwd_err(theirs, want) <= 1e-12, (dims, solvedim)
    assert ps.status_check()[1] == 0
