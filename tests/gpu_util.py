"""Helpers for the GPU parity tests: move seeded numpy problems to the device,
run the library through its C ABI, compare against the oracle."""
from __future__ import annotations

import numpy as np

import pentadsolver as ps

NAMES = ("ds", "dl", "d", "du", "dw", "x")

# Kernel selections exercised by the parity tests: (label, direction-specific
# algorithm name, pcr_lanes).  "transpose" only exists for x.
SELECTIONS = [
    ("auto", "auto", 0),
    ("naive", "naive", 0),
    ("pcr-p1", "thomas-pcr", 1),
    ("pcr-p2", "thomas-pcr", 2),
    ("transpose", "transpose", 0),
]


def to_dev(co: dict, device="cuda"):
    import torch

    return {k: torch.from_numpy(np.ascontiguousarray(co[k])).to(device) for k in NAMES}


def direction(ndim: int, solvedim: int) -> int:
    if solvedim == 0:
        return 0
    return 2 if solvedim == ndim - 1 else 1


def solve_dev(dv: dict, solvedim: int, dims=None, handle=None, buffer=None, stream=None,
              check_status: bool = True):
    """Solve through the C ABI; by default also require a clean status word
    afterwards -- the handle's own (no zero pivot, no timed-out wait)."""
    x = dv["x"]
    dims = ps.dims_of(x) if dims is None else list(dims)
    if buffer is None:
        buffer = ps.alloc_buffer(dims, solvedim, x.dtype, x.device)
    ps.gpsv_batch(dv["ds"], dv["dl"], dv["d"], dv["du"], dv["dw"], x, solvedim,
                  buffer=buffer, handle=handle, dims=dims, stream=stream)
    if check_status:
        st, bits = ps.status_check(stream=stream, handle=handle)
        assert bits == 0, f"device status bits {bits:#x} after solve along {solvedim}"
    return buffer


def fwd_err(x, ref) -> float:
    x = np.asarray(x, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.max(np.abs(ref))
    return float(np.max(np.abs(x - ref)) / (den if den > 0 else 1.0))


def allclose_ref(actual, expected, dtype):
    """test/catch_utils.hpp:19-22: per element rel 1e-13 or abs 1e-15 (FP64),
    rel 1e-5 or abs 1e-6 (FP32)."""
    rel, ab = (1e-13, 1e-15) if np.dtype(dtype) == np.float64 else (1e-5, 1e-6)
    a = np.asarray(actual, dtype=np.float64)
    e = np.asarray(expected, dtype=np.float64)
    diff = np.abs(a - e)
    ok = (diff <= ab) | (diff <= rel * np.abs(e))
    return bool(np.all(ok)), float(diff.max())
