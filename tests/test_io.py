"""CPU: output formats. The engine's VTK writer reproduces the reference's
write_vtk (include/lattice_io.hpp:386-451) byte for byte on the committed
fixtures (tests/golden/vtk_*.vtk, written by the reference build from
tests/golden/vtk_inputs.npz), given macroscopic fields computed in the
population precision as the reference computes them; restart files round-trip
and reject mismatched reads."""
import os

import numpy as np
import pytest

import lbcube as E
import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = {"D2Q9": (7, 5, 1), "D3Q19": (4, 3, 2)}


def macro_real(f, lattice, nx, ny, nz):
    """rho, u (population precision, exact) from the oracle, |u| = sqrt(u.u)
    with the squares added in ascending order in that precision."""
    rho, u = O.macro_fields(f, lattice, nx, ny, nz)
    dt = f.dtype.type
    rho, u = rho.astype(dt), u.astype(dt)
    s2 = u[0] * u[0]
    for d in range(1, u.shape[0]):
        s2 = s2 + u[d] * u[d]
    return rho, np.ascontiguousarray(u), np.sqrt(s2)


@pytest.mark.parametrize("lat", list(CASES))
@pytest.mark.parametrize("dn", ["float", "double"])
def test_vtk_matches_reference_fixture(tmp_path, lat, dn):
    nx, ny, nz = CASES[lat]
    f = np.load(os.path.join(GOLD, "vtk_inputs.npz"))[f"{lat}_{dn}"]
    rho, u, sp = macro_real(f, lat, nx, ny, nz)
    step = 42 + (dn == "double")
    path = str(tmp_path / f"lbm_{step:06d}.vtk")
    dims = 2 if lat == "D2Q9" else 3
    assert E.write_vtk_legacy(path, dims, nx, ny, nz, step, dn, rho, u, sp) == 0
    with open(path, "rb") as a, open(os.path.join(GOLD, f"vtk_{lat}_{dn}.vtk"), "rb") as b:
        assert a.read() == b.read()


def test_vtk_large_threaded(tmp_path):
    """Above the threading threshold the pieces are written in order."""
    n = 300 * 300
    rng = np.random.default_rng(1)
    rho = rng.random(n).astype(np.float32)
    u = rng.standard_normal((2, n)).astype(np.float32)
    sp = np.sqrt(u[0] * u[0] + u[1] * u[1])
    path = str(tmp_path / "big.vtk")
    assert E.write_vtk_legacy(path, 2, 300, 300, 1, 7, "float", rho, u, sp) == 0
    lines = open(path).read().splitlines()
    assert lines[4] == "DIMENSIONS 300 300 1" and lines[7] == f"POINT_DATA {n}"
    dens = np.array(lines[10:10 + n], dtype=np.float64)
    assert np.array_equal(dens, rho.astype(np.float64))
    vec = np.array([ln.split() for ln in lines[10 + n + 2 + n + 1:]], dtype=np.float64)
    assert vec.shape == (n, 3) and np.array_equal(vec[:, 1], u[1].astype(np.float64)) and not vec[:, 2].any()


def test_vtk_bad_arguments(tmp_path):
    a = np.zeros(4, np.float32)
    assert E.write_vtk_legacy(str(tmp_path / "x.vtk"), 4, 2, 2, 1, 0, "float", a, a, a) == E.IO_ERRORS["bad_argument"]
    assert E.write_vtk_legacy(str(tmp_path / "nodir" / "x.vtk"), 2, 2, 2, 1, 0, "float", a, np.zeros(8, np.float32),
                              a) == E.IO_ERRORS["open_failed"]


def test_restart_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    f = rng.random((19, 3, 4, 5)).astype(np.float64)
    path = str(tmp_path / "state.lbp")
    assert E.write_populations(path, "D3Q19", "double", 5, 4, 3, 1234, f) == 0
    assert os.path.getsize(path) == 64 + f.nbytes
    g = np.empty_like(f)
    rc, step = E.read_populations(path, "D3Q19", "double", 5, 4, 3, g)
    assert rc == 0 and step == 1234 and np.array_equal(f, g)
    assert E.read_populations(path, "D3Q19", "float", 5, 4, 3, g)[0] == E.IO_ERRORS["mismatch"]
    assert E.read_populations(path, "D3Q19", "double", 5, 4, 2, g)[0] == E.IO_ERRORS["mismatch"]
    with open(path, "r+b") as fh:
        fh.write(b"XXXX")
    assert E.read_populations(path, "D3Q19", "double", 5, 4, 3, g)[0] == E.IO_ERRORS["bad_file"]
    assert E.read_populations(str(tmp_path / "none"), "D3Q19", "double", 5, 4, 3, g)[0] == \
        E.IO_ERRORS["open_failed"]
