"""Generates tests/golden/reference_steps.npz from LB-Cube's own CPU path.

Runs the reference build (oracle/_ref/libref.so: the unmodified reference
headers compiled in place by `make -C oracle ref`) on small seeded states and
stores inputs and outputs, so the oracle and the engine can be checked against
the reference where its sources are not available. Regenerate with
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, ".."))

import _util as U  # noqa: E402
import oracle as O  # noqa: E402

SIZES = {"D2Q9": (7, 5, 1), "D3Q19": (6, 5, 4), "D3Q27": (5, 4, 3)}
OMEGA, OMEGA_C, K, STEPS = 1 / 0.6, 1 / 0.8, 0.07, 3


def main():
    if not O.REF.available:
        raise SystemExit("reference build oracle/_ref/libref.so missing: run make -C oracle ref")
    out = {}
    for lat, (nx, ny, nz) in SIZES.items():
        for dt, dn in ((np.float32, "float"), (np.float64, "double")):
            f = U.random_state(lat, nx, ny, nz, dt, seed=901)
            out[f"{lat}_{dn}_in"] = f
            for op in ("BGK", "TRT", "MRT", "RLBM"):
                out[f"{lat}_{dn}_{op}"] = O.step(f, lat, op, nx, ny, nz, OMEGA, steps=STEPS, lib=O.REF)
            sl = O.SCALAR_OF[lat]
            a = U.random_scalar(sl, nx, ny, nz, dt, seed=902)
            b = U.random_scalar(sl, nx, ny, nz, dt, seed=903)
            out[f"{lat}_{dn}_a_in"], out[f"{lat}_{dn}_b_in"] = a, b
            out[f"{lat}_{dn}_scalar"] = O.scalar_step(a, f, lat, nx, ny, nz, OMEGA_C, 1e-3, steps=STEPS, lib=O.REF)
            ra, rb = O.reaction_ab(a, b, f, lat, nx, ny, nz, OMEGA_C, K, steps=STEPS, lib=O.REF)
            out[f"{lat}_{dn}_react_a"], out[f"{lat}_{dn}_react_b"] = ra, rb
            out[f"{lat}_{dn}_stats"] = O.reactive_stats(a, b, sl, nx, ny, nz, K, lib=O.REF)
    np.savez_compressed(os.path.join(HERE, "reference_steps.npz"), **out)
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    main()
