"""GPU: device fluid diagnostics and the blow-up flag against the oracle.

Bars: max |u|, the non-finite count and the flag are exact (the per-cell
terms are computed in the population precision as the reference computes
them); total mass and kinetic energy are FP64 sums in another order than the
oracle's FP64 sums, relative error <= 1e-12. The fused step + diagnostics
writes the same populations as the plain step, bit for bit."""
import json
import math
import os

import numpy as np
import pytest
import torch

import _util as U
import oracle as O

pytestmark = pytest.mark.gpu

REALS = {"float": np.float32, "double": np.float64}
# vectorisable (even nx) and one-cell-kernel (odd nx) extents
SIZES = {"D2Q9": [(64, 20, 1), (37, 23, 1)], "D3Q19": [(32, 12, 9), (13, 11, 7)],
         "D3Q27": [(16, 6, 5), (9, 7, 5)]}


def _close(got, want):
    assert got[2] == want[2], (got, want)
    assert got[3] == want[3] and got[4] == want[4], (got, want)
    for k in (0, 1):
        assert abs(got[k] - want[k]) <= 1e-12 * abs(want[k]), (k, got, want)


def _scratch(engine, dev, lat, nx, ny, nz):
    nb = engine.diagnostics_partials_bytes(lat, nx, ny, nz)
    return torch.empty(nb, dtype=torch.uint8, device=dev), nb, torch.full((5,), -1.0, dtype=torch.float64,
                                                                          device=dev)


@pytest.mark.parametrize("lat", list(SIZES))
@pytest.mark.parametrize("real", list(REALS))
def test_diagnostics_match_oracle(engine, dev, lat, real):
    for k, (nx, ny, nz) in enumerate(SIZES[lat]):
        f = U.random_state(lat, nx, ny, nz, REALS[real], seed=40 + k, u_amp=0.05)
        part, nb, out = _scratch(engine, dev, lat, nx, ny, nz)
        t = torch.from_numpy(f).to(dev)
        for limit in (math.inf, 0.05):
            engine.check(engine.fluid_diagnostics_async(lat, real, t, nx, ny, nz, part, nb, out, limit))
            _close(out.cpu().numpy(), O.fluid_diagnostics64(f, lat, nx, ny, nz, limit))
        # the reference's own max (Real accumulators) is the same value
        assert out[2].item() == O.fluid_diagnostics(f, lat, nx, ny, nz)[2]


@pytest.mark.parametrize("lat", list(SIZES))
@pytest.mark.parametrize("real", list(REALS))
@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT", "RLBM"])
def test_step_diagnostics_fused(engine, dev, lat, real, op):
    for k, (nx, ny, nz) in enumerate(SIZES[lat]):
        f = U.random_state(lat, nx, ny, nz, REALS[real], seed=60 + k)
        cur = torch.from_numpy(f).to(dev)
        a, b = torch.empty_like(cur), torch.empty_like(cur)
        part, nb, out = _scratch(engine, dev, lat, nx, ny, nz)
        engine.check(engine.step_async(lat, real, op, cur, a, nx, ny, nz, 1 / 0.6))
        engine.check(engine.step_diagnostics_async(lat, real, op, cur, b, nx, ny, nz, 1 / 0.6, part, nb, out,
                                                   speed_limit=1.0))
        torch.cuda.synchronize()
        assert torch.equal(a, b), f"{lat} {real} {op} {nx}x{ny}x{nz}"
        _close(out.cpu().numpy(), O.fluid_diagnostics64(b.cpu().numpy(), lat, nx, ny, nz, 1.0))


def test_non_finite_cells_flagged(engine, dev):
    nx, ny, nz = 16, 6, 5
    f = U.random_state("D3Q19", nx, ny, nz, np.float32, seed=7)
    f[4, 33] = np.nan  # a NaN population: the cell's speed is NaN
    f[0, 90] = np.inf  # an infinite density: u = j / inf = 0, a finite speed; mass inf, KE NaN
    f[1, 200] = np.float32(3e38)
    f[2, 200] = np.float32(-3e38)  # finite density, overflowing momentum sum -> speed inf
    part, nb, out = _scratch(engine, dev, "D3Q19", nx, ny, nz)
    engine.check(engine.fluid_diagnostics_async("D3Q19", "float", torch.from_numpy(f).to(dev), nx, ny, nz,
                                                part, nb, out, 1.0))
    got, want = out.cpu().numpy(), O.fluid_diagnostics64(f, "D3Q19", nx, ny, nz, 1.0)
    assert got[3] == want[3] >= 2 and got[4] == want[4] == 1.0
    assert got[2] == want[2]  # NaN speeds skipped, an infinite one kept


def test_c1_diagnostics_every_step(engine, dev):
    """C1 (D3Q19 BGK FP64 64^3 Taylor-Green, tau 0.6) with the fused step:
    after 100 steps the diagnostics equal the reference build's log_diagnostics
    row (max |u| exactly; FP64 sums to 1e-12)."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden

    ref = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "c1_tgv64_fp64_bgk.json")))
    cur = torch.from_numpy(make_golden.tgv_c1()).to(dev)
    nxt = torch.empty_like(cur)
    part, nb, out = _scratch(engine, dev, "D3Q19", 64, 64, 64)
    for _ in range(100):
        engine.check(engine.step_diagnostics_async("D3Q19", "double", "BGK", cur, nxt, 64, 64, 64, 1 / 0.6,
                                                   part, nb, out, speed_limit=0.2))
        cur, nxt = nxt, cur
    got = out.cpu().numpy()
    want = ref["diagnostics_every_100"][1]
    assert got[2] == want[2] and got[3] == 0 and got[4] == 0
    for k in (0, 1):
        assert abs(got[k] - want[k]) <= 1e-12 * abs(want[k])
