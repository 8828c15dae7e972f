"""GPU: macroscopic output fields computed on the device are bit-identical to
the reference's per-cell reconstruction (compute_macro_state, sqrt(u.u) in
the population precision), and the VTK file written from them equals the
reference build's write_vtk output byte for byte."""
import os

import numpy as np
import pytest
import torch

import _util as U
import lbcube as E
import oracle as O
from test_io import CASES, GOLD, macro_real

pytestmark = pytest.mark.gpu

SIZES = {"D2Q9": (37, 23, 1), "D3Q19": (13, 11, 7), "D3Q27": (9, 7, 5)}
REALS = {"float": np.float32, "double": np.float64}


def device_macro(lat, dn, f, nx, ny, nz, dev):
    t = torch.from_numpy(f).to(dev)
    n = f.shape[1]
    D = O.D_OF[lat]
    dt = t.dtype
    rho = torch.empty(n, dtype=dt, device=dev)
    u = torch.empty((D, n), dtype=dt, device=dev)
    sp = torch.empty(n, dtype=dt, device=dev)
    E.check(E.macro_fields_async(lat, dn, t, nx, ny, nz, rho, u, sp))
    torch.cuda.synchronize()
    return rho.cpu().numpy(), u.cpu().numpy(), sp.cpu().numpy()


@pytest.mark.parametrize("lat", list(SIZES))
@pytest.mark.parametrize("dn", list(REALS))
def test_macro_fields_bitwise(engine, dev, lat, dn):
    nx, ny, nz = SIZES[lat]
    f = U.random_state(lat, nx, ny, nz, REALS[dn], seed=70, u_amp=0.05)
    got = device_macro(lat, dn, f, nx, ny, nz, dev)
    want = macro_real(f, lat, nx, ny, nz)
    for g, w in zip(got, want):
        assert U.same_bits(g, w)


@pytest.mark.parametrize("sl", ["D2Q5", "D3Q7"])
def test_scalar_concentration(engine, dev, sl):
    nx, ny, nz = (19, 6, 1) if sl == "D2Q5" else (7, 6, 5)
    g = U.random_scalar(sl, nx, ny, nz, np.float32, seed=4)
    t = torch.from_numpy(g).to(dev)
    c = torch.empty(g.shape[1], dtype=torch.float32, device=dev)
    E.check(E.macro_fields_async(sl, "float", t, nx, ny, nz, c))
    want, _ = O.macro_fields(g, sl, nx, ny, nz)
    assert np.array_equal(c.cpu().numpy().astype(np.float64), want)
    assert E.macro_fields_async(sl, "float", t, nx, ny, nz, c, velocity=c) == E.cudaErrorInvalidValue
    assert E.macro_fields_async(sl, "float", t, nx, ny, nz, None) == E.cudaErrorInvalidValue


@pytest.mark.parametrize("lat", list(CASES))
@pytest.mark.parametrize("dn", ["float", "double"])
def test_vtk_from_device_fields(engine, dev, tmp_path, lat, dn):
    nx, ny, nz = CASES[lat]
    f = np.load(os.path.join(GOLD, "vtk_inputs.npz"))[f"{lat}_{dn}"]
    rho, u, sp = device_macro(lat, dn, f, nx, ny, nz, dev)
    step = 42 + (dn == "double")
    path = str(tmp_path / f"lbm_{step:06d}.vtk")
    assert E.write_vtk_legacy(path, 2 if lat == "D2Q9" else 3, nx, ny, nz, step, dn, rho, u, sp) == 0
    with open(path, "rb") as a, open(os.path.join(GOLD, f"vtk_{lat}_{dn}.vtk"), "rb") as b:
        assert a.read() == b.read()
