"""Committed reference outputs (tests/golden/reference_steps.npz, made by
tests/golden/make_golden.py from the reference's own CPU path) against the
oracle (CPU) and against the engine (GPU). Step, scalar and statistics outputs
are compared bit for bit; the reaction (exp) to the stated tolerances."""
import os

import numpy as np

import _util as U
import pytest

import oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_steps.npz"))
SIZES = {"D2Q9": (7, 5, 1), "D3Q19": (6, 5, 4), "D3Q27": (5, 4, 3)}
OMEGA, OMEGA_C, K, STEPS = 1 / 0.6, 1 / 0.8, 0.07, 3
CASES = [(lat, dn) for lat in SIZES for dn in ("float", "double")]


@pytest.mark.parametrize("lat,dn", CASES)
def test_oracle_matches_reference_fixtures(lat, dn):
    nx, ny, nz = SIZES[lat]
    f = G[f"{lat}_{dn}_in"]
    for op in ("BGK", "TRT", "MRT", "RLBM"):
        assert U.same_bits(O.step(f, lat, op, nx, ny, nz, OMEGA, steps=STEPS), G[f"{lat}_{dn}_{op}"]), op
    a, b = G[f"{lat}_{dn}_a_in"], G[f"{lat}_{dn}_b_in"]
    assert U.same_bits(O.scalar_step(a, f, lat, nx, ny, nz, OMEGA_C, 1e-3, steps=STEPS), G[f"{lat}_{dn}_scalar"])
    ra, rb = O.reaction_ab(a, b, f, lat, nx, ny, nz, OMEGA_C, K, steps=STEPS)
    assert U.same_bits(ra, G[f"{lat}_{dn}_react_a"]) and U.same_bits(rb, G[f"{lat}_{dn}_react_b"])
    assert U.same_bits(O.reactive_stats(a, b, O.SCALAR_OF[lat], nx, ny, nz, K), G[f"{lat}_{dn}_stats"])


@pytest.mark.gpu
@pytest.mark.parametrize("lat,dn", CASES)
def test_engine_matches_reference_fixtures(engine, dev, lat, dn):
    import torch

    nx, ny, nz = SIZES[lat]
    f = G[f"{lat}_{dn}_in"]
    for op in ("BGK", "TRT", "MRT", "RLBM"):
        cur = torch.from_numpy(f.copy()).to(dev)
        nxt = torch.empty_like(cur)
        for _ in range(STEPS):
            engine.check(engine.launch_step_gpu(lat, dn, op, cur, nxt, nx, ny, nz, OMEGA))
            cur, nxt = nxt, cur
        torch.cuda.synchronize()
        assert U.same_bits(cur.cpu().numpy(), G[f"{lat}_{dn}_{op}"]), op
    tf = torch.from_numpy(f.copy()).to(dev)
    ta = torch.from_numpy(G[f"{lat}_{dn}_a_in"].copy()).to(dev)
    tb = torch.from_numpy(G[f"{lat}_{dn}_b_in"].copy()).to(dev)
    na, nb = torch.empty_like(ta), torch.empty_like(tb)
    for _ in range(STEPS):
        engine.check(engine.launch_reaction_AB_gpu(lat, dn, ta, na, tb, nb, tf, nx, ny, nz, OMEGA_C, K))
        ta, na, tb, nb = na, ta, nb, tb
    torch.cuda.synchronize()
    tol = 1e-13 if dn == "double" else 1e-5
    for got, key in ((ta, "react_a"), (tb, "react_b")):
        want = G[f"{lat}_{dn}_{key}"]
        assert np.linalg.norm(got.cpu().numpy() - want) / np.linalg.norm(want) <= tol


C1 = os.path.join(os.path.dirname(__file__), "golden", "c1_tgv64_fp64_bgk.json")


def _c1_initial():
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden

    return make_golden.tgv_c1()


def test_oracle_c1_first_100_steps():
    """C1 (D3Q19 BGK FP64 64^3 Taylor-Green): the oracle's (mass, KE, max|u|)
    after 0 and 100 steps equal the reference build's, bit for bit."""
    import json

    want = json.load(open(C1))["diagnostics_every_100"]
    f = _c1_initial()
    assert O.fluid_diagnostics(f, "D3Q19", 64, 64, 64).tolist() == want[0]
    f = O.step(f, "D3Q19", "BGK", 64, 64, 64, 1 / 0.6, steps=100)
    assert O.fluid_diagnostics(f, "D3Q19", 64, 64, 64).tolist() == want[1]


@pytest.mark.gpu
def test_engine_c1_fingerprint(engine, dev):
    """C1 on the engine: 1000 steps through the drop-in launcher; every 100
    steps the diagnostics equal the reference build's and the final
    populations have the reference's SHA-256."""
    import hashlib
    import json

    import torch

    ref = json.load(open(C1))
    cur = torch.from_numpy(_c1_initial()).to(dev)
    nxt = torch.empty_like(cur)
    for block in range(1, ref["steps"] // 100 + 1):
        for _ in range(100):
            engine.check(engine.launch_step_gpu("D3Q19", "double", "BGK", cur, nxt, 64, 64, 64, 1 / 0.6))
            cur, nxt = nxt, cur
        f = cur.cpu().numpy()
        assert O.fluid_diagnostics(f, "D3Q19", 64, 64, 64).tolist() == ref["diagnostics_every_100"][block], block
    assert hashlib.sha256(f.tobytes()).hexdigest() == ref["sha256_final"]
