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


def tgv_c1(n=64, u0=0.05):
    """The C1 initial field: D3Q19 Taylor-Green u = u0 (sin kx cos ky cos kz,
    -cos kx sin ky cos kz, 0), rho = 1, k = 2 pi / n. Built from 1-D tables of
    glibc sin/cos (math module) and IEEE products, so every machine running
    this image reproduces the same bits."""
    import math

    k = 2 * math.pi / n
    s1 = np.array([math.sin(k * i) for i in range(n)])
    c1 = np.array([math.cos(k * i) for i in range(n)])
    ux = u0 * s1[None, None, :] * c1[None, :, None] * c1[:, None, None]
    uy = -u0 * c1[None, None, :] * s1[None, :, None] * c1[:, None, None]
    u = np.stack([ux, uy, np.zeros_like(ux)]).reshape(3, -1)
    return O.init_equilibrium("D3Q19", np.ones(n ** 3), u, n, n, n)


def c1_fingerprint(steps=1000, every=100, tau=0.6):
    """C1 run on the reference CPU path: SHA-256 of the final populations and
    the (mass, KE, max |u|) series every `every` steps."""
    import hashlib

    f = tgv_c1()
    series = [O.fluid_diagnostics(f, "D3Q19", 64, 64, 64).tolist()]
    for _ in range(steps // every):
        f = O.step(f, "D3Q19", "BGK", 64, 64, 64, 1 / tau, steps=every, lib=O.REF)
        series.append(O.fluid_diagnostics(f, "D3Q19", 64, 64, 64).tolist())
    return {"workload": "D3Q19 BGK FP64 64^3 Taylor-Green u0 0.05 rho 1, tau 0.6",
            "steps": steps, "sha256_final": hashlib.sha256(f.tobytes()).hexdigest(),
            "diagnostics_every_100": series}


VTK_CASES = {"D2Q9": (7, 5, 1), "D3Q19": (4, 3, 2)}


def make_vtk_golden():
    """The reference's write_vtk text for seeded states (legacy ASCII VTK,
    lattice_io.hpp:386-451), with the populations it was written from."""
    import tempfile

    inputs = {}
    with tempfile.TemporaryDirectory() as tmp:
        for lat, (nx, ny, nz) in VTK_CASES.items():
            for k, (dn, dt) in enumerate((("float", np.float32), ("double", np.float64))):
                f = U.random_state(lat, nx, ny, nz, dt, seed=300 + k, u_amp=0.05)
                inputs[f"{lat}_{dn}"] = f
                text = O.reference_vtk(f, lat, nx, ny, nz, 42 + k, tmp)
                with open(os.path.join(HERE, f"vtk_{lat}_{dn}.vtk"), "wb") as fh:
                    fh.write(text)
    np.savez_compressed(os.path.join(HERE, "vtk_inputs.npz"), **inputs)


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
    import json

    with open(os.path.join(HERE, "c1_tgv64_fp64_bgk.json"), "w") as fh:
        json.dump(c1_fingerprint(), fh, indent=1)
    print("wrote the C1 fingerprint")
    make_vtk_golden()
    print("wrote the VTK fixtures")


if __name__ == "__main__":
    main()
