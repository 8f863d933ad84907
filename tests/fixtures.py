"""Test inputs: golden fixture loading and the seeded synthetic generators.

Array convention: numpy C order with the LAST numpy axis equal to the
reference's ``t_dims[0]`` (the contiguous x axis).  ``dims`` lists are fastest
first, exactly as the reference API takes them.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"
NAMES = ("ds", "dl", "d", "du", "dw", "x", "u", "u_float")

# Reference fixture families and their number of solve dimensions
# (test/gen_testcases.py:126-131; the tests of test/cpu/singlenode/tests.cpp).
FAMILIES = {
    "one_dim_small": 1,
    "one_dim_large": 1,
    "two_dim_small": 2,
    "two_dim_large": 2,
    "three_dim_large": 3,
}


def rotate(base: dict, k: int) -> dict:
    """The solvedim-k fixture from the solvedim-0 one.

    ``test/gen_testcases.py:113-123`` writes file k after k rotations of the
    numpy axes by ``transpose(1, .., n-1, 0)``; the solve axis (originally the
    last numpy axis) then sits at reference dimension k.
    """
    out = {"solvedim": k}
    nd = base["ds"].ndim
    perm = tuple(list(range(1, nd)) + [0])
    for name in NAMES:
        a = base[name]
        for _ in range(k):
            a = a.transpose(perm)
        out[name] = np.ascontiguousarray(a)
    out["dims"] = [int(v) for v in reversed(out["ds"].shape)]
    return out


def load_family(fam: str) -> dict:
    z = np.load(GOLDEN / f"{fam}.npz")
    base = {name: z[name] for name in NAMES}
    base["dims"] = [int(v) for v in z["dims"]]
    base["solvedim"] = 0
    return base


def load_fixture(fam: str, solvedim: int) -> dict:
    return rotate(load_family(fam), solvedim)


def all_fixture_cases():
    for fam, nd in FAMILIES.items():
        for k in range(nd):
            yield fam, k


def random_dominant(dims, seed: int, dtype=np.float64, zero_axis=None) -> dict:
    """Seeded random diagonally dominant coefficients (the 64^3 parity config).

    Per point the off-diagonals ds (i-2), dl (i-1), du (i+1), dw (i+2) are
    U(-1,1), the diagonal is |ds|+|dl|+|du|+|dw| + U(1,2) and the RHS is
    U(-1,1), drawn from numpy's PCG64 with ``seed``.  Values are drawn in FP64
    and rounded once for FP32.  With ``zero_axis=k`` the entries that lie
    outside the lines along reference dimension k are zeroed (every solver
    ignores them, so this changes no result).
    """
    rng = np.random.default_rng(seed)
    shape = tuple(int(v) for v in reversed(dims))
    ds = rng.uniform(-1.0, 1.0, shape)
    dl = rng.uniform(-1.0, 1.0, shape)
    du = rng.uniform(-1.0, 1.0, shape)
    dw = rng.uniform(-1.0, 1.0, shape)
    d = np.abs(ds) + np.abs(dl) + np.abs(du) + np.abs(dw) + rng.uniform(1.0, 2.0, shape)
    x = rng.uniform(-1.0, 1.0, shape)
    out = {"ds": ds, "dl": dl, "d": d, "du": du, "dw": dw, "x": x}
    if zero_axis is not None:
        zero_out_of_range(out, zero_axis)
    return {k: np.ascontiguousarray(v.astype(dtype)) for k, v in out.items()}


def zero_out_of_range(co: dict, axis: int) -> None:
    """Zero ds at rows 0,1; dl at row 0; du at row n-1; dw at rows n-2, n-1."""
    nd = co["ds"].ndim
    ax = nd - 1 - axis  # numpy axis of reference dimension `axis`

    def sl(idx):
        s = [slice(None)] * nd
        s[ax] = idx
        return tuple(s)

    co["ds"][sl(slice(0, 2))] = 0
    co["dl"][sl(slice(0, 1))] = 0
    co["du"][sl(slice(-1, None))] = 0
    co["dw"][sl(slice(-2, None))] = 0


def adi_constant(dims, r: float = 0.5, dtype=np.float64, seed: int = 2024) -> dict:
    """Constant-coefficient ADI problem: ds=dw=-r/12, dl=du=16r/12, d=1+30r/12.

    The initial field is U(-1,1) from ``seed``.  Out-of-range entries are left
    at the constants: every solver ignores them.
    """
    shape = tuple(int(v) for v in reversed(dims))
    rng = np.random.default_rng(seed)
    out = {
        "ds": np.full(shape, -r / 12.0),
        "dl": np.full(shape, 16.0 * r / 12.0),
        "d": np.full(shape, 1.0 + 30.0 * r / 12.0),
        "du": np.full(shape, 16.0 * r / 12.0),
        "dw": np.full(shape, -r / 12.0),
        "x": rng.uniform(-1.0, 1.0, shape),
    }
    return {k: np.ascontiguousarray(v.astype(dtype)) for k, v in out.items()}


def load_refrun(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz")
    return {k: z[k] for k in z.files}


REFRUNS = ("refrun_16cube", "refrun_20x12x9", "refrun_33x7x6")
