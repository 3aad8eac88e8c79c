"""Generates the golden fixtures of tests/golden/ from the reference's own
step loop (oracle/_ref/felis_ref: the reference's unmodified sources compiled
with the MPI/GSL stand-ins of oracle/ref_shim/).

Each fixture is the result of a whole run of the reference from the
initial state its own loader makes (GSL_RNG_SEED as named; the product's
loader gives the same bits, tests/test_ref_pin.py), stored subsampled so
that it stays small:

  ref_config1.npz        config 1 complete: Static, 8192 quiet-start
                         particles, 102 x 102 grid, 1 MW seed, 1539 steps
  ref_config2_prefix.npz config 2 (Time_Dependent SASE, 8192 particles per
                         slice, shot noise, no seed, 1539 steps) on its first
                         2 slices: slippage carries radiation only from slice
                         s-1 to s (solveField.cpp:19-47), so slices 1..k of
                         the 1024-slice run evolve exactly as a k-slice run

Contents: 'input' (the input file text), 'seed', 'energy' (iterations x 2H:
sum |Ux_h|^2, sum |Uy_h|^2 of updateTotalEnergy), 'pick' (particle indices)
with the six final particle columns at those indices, 'field_x'/'field_y'
(final planes of slices 1..S of harmonic 1, every 3rd cell in x and y).

Run from the repository root: python tests/golden/make_ref_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refrun  # noqa: E402
from felis_b200 import workloads  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
PREFIX_SLICES = 2
PARTICLE_STRIDE = 16
CELL_STRIDE = 3

FIXTURES = {
    "ref_config1.npz": (dict(kind="static"), 1),
    "ref_config2_prefix.npz": (dict(kind="sase", slices=PREFIX_SLICES), 2),
}


def subsample(res: dict) -> dict:
    b = res["final"]["particles"][0]
    n = b["x"].size
    pick = np.arange(0, n, PARTICLE_STRIDE, dtype=np.int64)
    out = {k: b[k][pick] for k in refrun.KEYS}
    out["pick"] = pick
    out["offsets"] = b["offsets"]
    out["field_x"] = res["final"]["Ux"][0][1:-1, ::CELL_STRIDE, ::CELL_STRIDE]
    out["field_y"] = res["final"]["Uy"][0][1:-1, ::CELL_STRIDE, ::CELL_STRIDE]
    out["energy"] = np.stack([res["energyX"], res["energyY"]], axis=2).reshape(res["energyX"].shape[0], -1)
    return out


def main():
    if not refrun.build():
        raise SystemExit("oracle/_ref is not built and the reference sources are absent")
    for name, (kw, seed) in FIXTURES.items():
        d = tempfile.mkdtemp(prefix="felis_golden_")
        path = workloads.write_input(os.path.join(d, "case.inp"), **kw)
        with open(path) as f:
            text = f.read()
        res = refrun.run(path, seed=seed)
        data = subsample(res)
        np.savez_compressed(os.path.join(HERE, name), input=np.array(text), seed=np.array(seed),
                            particle_stride=np.array(PARTICLE_STRIDE), cell_stride=np.array(CELL_STRIDE), **data)
        print(name, "energy[-1]", data["energy"][-1], "particles", data["offsets"][-1])


if __name__ == "__main__":
    main()
