"""Generates the golden fixtures under tests/golden/ from LB-Cube's own CPU path.

Runs the reference build (oracle/_ref/libref.so: the unmodified reference
headers compiled in place by `make -C oracle ref`) on small seeded states and
stores inputs and outputs, so the oracle and the engine can be checked against
the reference where its sources are not available. Regenerate with
    python tests/golden/make_golden.py          # the small fixtures (a minute)
    python tests/golden/make_golden.py --c3     # the 1024^2 reactive-mixing run
                                                # (about an hour on one core)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, ".."))
sys.path.insert(0, os.path.join(HERE, "..", "..", "lb-cube_b200"))

import _util as U  # noqa: E402
import oracle as O  # noqa: E402
import workloads as W  # noqa: E402

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


C3_FILE = os.path.join(HERE, "c3_shear1024_mrt.npz")


def concentration(g, q):
    """C = sum of the scalar populations, in ascending order (FP64)."""
    g = np.asarray(g, np.float64).reshape(q, -1)
    c = g[0].copy()
    for i in range(1, q):
        c += g[i]
    return c


def c3_reactive_mixing(n=1024, steps=20000, every=10, out=C3_FILE):
    """The reactive-mixing configuration on the reference CPU path: D2Q9 MRT
    fluid (tau 0.6) on the double shear layer of workloads.reactive_shear_layer
    and two D2Q5 species reacting A + B -> C (Pe 1000, Da 1, L = n), stepped
    as src/simulate_reaction.cpp:515-555 steps it (step_cpu, then
    step_reaction_AB with the post-step fluid), with compute_reactive_stats
    (lattice_io.hpp:256-338) at step 0 and every `every` steps, as
    log_reactive_diagnostics records it.

    Stores: the workload's 1-D tables; the statistics rows as the reference
    computes them (sums in FP32) and the same rows with FP64 sums over the
    reference's fields; SHA-256 of the final fluid, A and B populations; the
    final concentrations' FP64 row and column sums and a stride-8 subsample."""
    import hashlib
    import time

    w = W.reactive_shear_layer(n)
    omega, omega_c, k = 1.0 / w["tau"], 1.0 / w["tau_c"], w["k"]
    f = O.init_equilibrium("D2Q9", w["rho"], w["u"], n, n, 1, np.float32)
    a = O.init_equilibrium("D2Q5", w["a0"], w["u"], n, n, 1, np.float32)
    b = O.init_equilibrium("D2Q5", w["b0"], w["u"], n, n, 1, np.float32)
    init_sha = hashlib.sha256(f.tobytes() + a.tobytes() + b.tobytes()).hexdigest()

    def stats_rows(a_, b_):
        return (O.reactive_stats(a_, b_, "D2Q5", n, n, 1, k, lib=O.REF),
                O.reactive_stats(a_, b_, "D2Q5", n, n, 1, k, accumulate_f64=True))

    r32, r64 = stats_rows(a, b)
    rows_ref, rows_f64 = [r32], [r64]
    t0 = time.time()
    for s in range(steps // every):
        f, a, b = O.coupled_reaction(f, a, b, "D2Q9", "MRT", n, n, 1, omega, omega_c, k, steps=every,
                                     lib=O.REF)
        r32, r64 = stats_rows(a, b)
        rows_ref.append(r32)
        rows_f64.append(r64)
        if (s + 1) % 100 == 0:
            print(f"C3: step {(s + 1) * every} of {steps}, {time.time() - t0:.0f} s", flush=True)
    ca, cb = concentration(a, 5).reshape(n, n), concentration(b, 5).reshape(n, n)
    np.savez_compressed(
        out, n=n, steps=steps, every=every, tau=w["tau"], tau_c=w["tau_c"], k=k, seed=W.SHEAR_SEED,
        ux_row=w["tables"]["ux_row"], cos_col=w["tables"]["cos_col"], init_sha256=init_sha,
        stats_reference=np.array(rows_ref), stats_f64=np.array(rows_f64),
        fluid_sha256=hashlib.sha256(f.tobytes()).hexdigest(),
        a_sha256=hashlib.sha256(a.tobytes()).hexdigest(), b_sha256=hashlib.sha256(b.tobytes()).hexdigest(),
        ca_rows=ca.sum(axis=1), ca_cols=ca.sum(axis=0), cb_rows=cb.sum(axis=1), cb_cols=cb.sum(axis=0),
        ca_sub=ca[::8, ::8].astype(np.float32), cb_sub=cb[::8, ::8].astype(np.float32),
        ca_l2=np.linalg.norm(ca), cb_l2=np.linalg.norm(cb))
    print(f"wrote {out}: {len(rows_ref)} statistics rows in {time.time() - t0:.0f} s")


def main():
    if "--c3" in sys.argv:
        steps = int(sys.argv[sys.argv.index("--c3") + 1]) if len(sys.argv) > sys.argv.index("--c3") + 1 else 20000
        return c3_reactive_mixing(steps=steps)
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
