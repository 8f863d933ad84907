#!/usr/bin/env python3
"""Regenerate the committed golden fixtures under tests/golden/.

Run here (it needs the reference tree, which the GPU box does not have):

    python tests/golden/make_golden.py [--ref REFERENCE_TREE]

(default: $PENTA_REFERENCE_DIR, else /root/reference)

1. Reference fixtures.  Runs the reference's own generator
   ``test/gen_testcases.py`` (numpy seed 1, scipy ``solve_banded``) in a
   temporary directory, parses every text file it writes with the reference's
   format (``include/util/mesh.hpp:51-80``: ``ndims solvedim`` / dims fastest
   first / ds dl d du dw x u u_float), checks the regenerated files against the
   ones the reference ships in ``test/cpu/singlenode/files`` (inputs identical,
   solutions within 1e-14), and stores each family once as ``<family>.npz`` in
   its solvedim-0 layout.  The loader in ``tests/fixtures.py`` rebuilds the
   solvedim-k files with the generator's own axis rotation
   (``gen_testcases.py:113-123``); this script checks that it does.  The 3-D
   family is the one the reference does not ship (``.MISSING_LARGE_BLOBS``).

2. Reference-run fixtures.  Seeded random diagonally dominant grids (off-
   diagonals U(-1,1), diagonal sum|off| + U(1,2), RHS U(-1,1)) solved along x,
   then y, then z by the reference's compiled CPU solvers (``oracle/_ref``):
   the scalar ``pentad_orig_cpu.cpp`` and, where its vector width divides dims[0], the AVX2
   ``pentad_cpu.cpp``.  Stored with the state after each axis.
"""
from __future__ import annotations

import argparse
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "tests"))

from oracle import oracle  # noqa: E402
import fixtures  # noqa: E402

FAMILIES = {
    "one_dim_small": 1,
    "one_dim_large": 1,
    "two_dim_small": 2,
    "two_dim_large": 2,
    "three_dim_large": 3,
}


def parse_fixture(path: Path) -> dict:
    """Parse one reference fixture file (mesh.hpp:51-80 format)."""
    toks = path.read_text().split()
    ndims, solvedim = int(toks[0]), int(toks[1])
    dims = [int(t) for t in toks[2:2 + ndims]]
    n = int(np.prod(dims))
    vals = np.array([float(t) for t in toks[2 + ndims:]], dtype=np.float64)
    assert vals.size == 8 * n, (path, vals.size, n)
    names = ["ds", "dl", "d", "du", "dw", "x", "u", "u_float"]
    out = {"dims": dims, "solvedim": solvedim}
    shape = tuple(reversed(dims))
    for k, name in enumerate(names):
        out[name] = vals[k * n:(k + 1) * n].reshape(shape)
    return out


def make_reference_fixtures(ref: Path) -> None:
    gen = ref / "test" / "gen_testcases.py"
    shipped = ref / "test" / "cpu" / "singlenode" / "files"
    with tempfile.TemporaryDirectory() as tmp:
        shutil.copy(gen, Path(tmp) / "gen_testcases.py")
        subprocess.run([sys.executable, "gen_testcases.py"], cwd=tmp, check=True,
                       stdout=subprocess.DEVNULL)
        for fam, nd in FAMILIES.items():
            files = {k: parse_fixture(Path(tmp) / f"{fam}_solve{k}") for k in range(nd)}
            base = files[0]
            # the rotation the loader applies must reproduce every solvedim file
            for k in range(nd):
                rebuilt = fixtures.rotate(base, k)
                got = files[k]
                assert rebuilt["dims"] == got["dims"] and rebuilt["solvedim"] == got["solvedim"]
                for name in ("ds", "dl", "d", "du", "dw", "x", "u", "u_float"):
                    assert np.array_equal(rebuilt[name], got[name]), (fam, k, name)
                ship = shipped / f"{fam}_solve{k}"
                if ship.exists():
                    s = parse_fixture(ship)
                    for name in ("ds", "dl", "d", "du", "dw", "x"):
                        assert np.array_equal(s[name], got[name]), (fam, k, name)
                    du = np.max(np.abs(s["u"] - got["u"]))
                    assert du <= 1e-14, (fam, k, du)
                    print(f"  {fam}_solve{k}: matches the shipped file (max |du| {du:.1e})")
            np.savez_compressed(HERE / f"{fam}.npz", dims=np.array(base["dims"]),
                                **{k: base[k] for k in ("ds", "dl", "d", "du", "dw",
                                                       "x", "u", "u_float")})
            print(f"wrote {fam}.npz")


def make_reference_runs() -> None:
    cases = [
        ("refrun_16cube", (16, 16, 16), 20231),
        ("refrun_20x12x9", (20, 12, 9), 777),
        ("refrun_33x7x6", (33, 7, 6), 4242),
    ]
    for name, dims, seed in cases:
        out = {"dims": np.array(dims)}
        for dt, tag in ((np.float64, "d"), (np.float32, "s")):
            co = fixtures.random_dominant(dims, seed, dt)
            out.update({f"{k}_{tag}": co[k] for k in ("ds", "dl", "d", "du", "dw", "x")})
            for which in ("orig", "simd"):
                if which == "simd" and not oracle.simd_ok(dims, dt):
                    continue
                x = co["x"].copy()
                for axis in range(3):
                    oracle.ref_solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"],
                                     x, axis, which=which)
                    out[f"after{axis}_{which}_{tag}"] = x.copy()
            # the restatement must agree bit for bit with the compiled reference
            xo = co["x"].copy()
            for axis in range(3):
                oracle.solve(co["ds"], co["dl"], co["d"], co["du"], co["dw"], xo, axis)
                assert np.array_equal(xo, out[f"after{axis}_orig_{tag}"]), (name, tag, axis)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"wrote {name}.npz")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=str(oracle.reference_dir()))
    args = ap.parse_args()
    make_reference_fixtures(Path(args.ref))
    make_reference_runs()


if __name__ == "__main__":
    main()
