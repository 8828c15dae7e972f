"""Committed reference outputs (tests/golden/reference_steps.npz, made by
tests/golden/make_golden.py from the reference's own CPU path) against the
oracle (CPU) and against the engine (GPU). Step, scalar and statistics outputs
are compared bit for bit; the reaction (exp) to the stated tolerances."""
import os

import numpy as np
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
        assert np.array_equal(O.step(f, lat, op, nx, ny, nz, OMEGA, steps=STEPS), G[f"{lat}_{dn}_{op}"]), op
    a, b = G[f"{lat}_{dn}_a_in"], G[f"{lat}_{dn}_b_in"]
    assert np.array_equal(O.scalar_step(a, f, lat, nx, ny, nz, OMEGA_C, 1e-3, steps=STEPS), G[f"{lat}_{dn}_scalar"])
    ra, rb = O.reaction_ab(a, b, f, lat, nx, ny, nz, OMEGA_C, K, steps=STEPS)
    assert np.array_equal(ra, G[f"{lat}_{dn}_react_a"]) and np.array_equal(rb, G[f"{lat}_{dn}_react_b"])
    assert np.array_equal(O.reactive_stats(a, b, O.SCALAR_OF[lat], nx, ny, nz, K), G[f"{lat}_{dn}_stats"])


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
        assert np.array_equal(cur.cpu().numpy(), G[f"{lat}_{dn}_{op}"]), op
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
