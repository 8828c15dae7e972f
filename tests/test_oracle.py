"""CPU: the oracle (oracle/lbm_oracle.c) pinned against the reference.

1. Golden vectors and known-answer tests from LB-Cube's own suite
   (tests/test_validation.cpp), rerun on the oracle with the same inputs and
   tolerances.
2. Bit-for-bit agreement with the reference's own CPU path compiled from its
   unmodified headers (oracle/_ref/libref.so), when that build is present.
"""
import math

import numpy as np
import pytest

import _util as U
import oracle as O

LATS = ("D2Q9", "D3Q19", "D3Q27")
OPS = ("BGK", "TRT", "MRT", "RLBM")
DTYPES = (np.float32, np.float64)
SMALL = {"D2Q9": (7, 5, 1), "D3Q19": (6, 5, 4), "D3Q27": (5, 4, 3)}

needs_ref = pytest.mark.skipif(not O.REF.available, reason="reference build oracle/_ref not present")


# --- golden vectors: MRT transform identities -------------------------------
def test_mrt_d2q9_identity():
    """MRT_D2Q9_Transformation_Identity (tests/test_validation.cpp:1532-1548): EXPECT_DOUBLE_EQ."""
    f = 1.125 * np.arange(1, 10, dtype=np.float64)
    back = O.mrt_populations("D2Q9", O.mrt_moments("D2Q9", f))
    ulp = np.abs(np.nextafter(f, np.inf) - f)
    assert np.all(np.abs(back - f) <= 4 * ulp)


@pytest.mark.parametrize("lat,q", [("D3Q19", 19), ("D3Q27", 27)])
def test_mrt_3d_identity(lat, q):
    """MRT_D3Q19/D3Q27_Transformation_Identity (test_validation.cpp:1550-1582): 1e-12."""
    f = 0.01 * np.arange(1, q + 1, dtype=np.float64)
    back = O.mrt_populations(lat, O.mrt_moments(lat, f))
    assert np.max(np.abs(back - f)) <= 1e-12


def test_mrt_moment_zero_is_density():
    rng = np.random.default_rng(3)
    for lat, q in (("D2Q9", 9), ("D3Q19", 19), ("D3Q27", 27)):
        f = rng.uniform(0, 1, q)
        assert math.isclose(O.mrt_moments(lat, f)[0], f.sum(), rel_tol=1e-15)


# --- known-answer tests ------------------------------------------------------
def test_mass_conservation_d3q19():
    """MassConservationD3Q19Cpu (test_validation.cpp:1283-1303): BGK, omega = 1,
    seeded rho in U[0.95, 1.05], u in U[-0.01, 0.01]; mass within 1024 eps M.
    (16^3 here instead of 32^3 to keep the CPU suite short.)"""
    n, steps = 16, 100
    rng = np.random.default_rng(0x5EED1234)
    rho = rng.uniform(0.95, 1.05, n ** 3)
    u = rng.uniform(-0.01, 0.01, (3, n ** 3))
    f = O.init_equilibrium("D3Q19", rho, u, n, n, n)
    m0 = math.fsum(f.ravel())
    g = O.step(f, "D3Q19", "BGK", n, n, n, 1.0, steps=steps)
    assert abs(math.fsum(g.ravel()) - m0) <= np.finfo(np.float64).eps * m0 * 1024


@pytest.mark.parametrize("op", ["BGK", "TRT", "MRT"])
def test_taylor_green_2d_decay(op):
    """TaylorGreenVortex_{BGK,TRT,MRT} (test_validation.cpp:576-602, :1336-1352):
    D2Q9 64^2, u0 = 0.01, tau = 0.8, 1000 steps; KE vs exp(-4 nu k^2 t) within 1e-5."""
    n, steps, u0, tau, cs2 = 64, 1000, 0.01, 0.8, 1.0 / 3.0
    k = 2 * math.pi / n
    nu = cs2 * (tau - 0.5)
    x = np.arange(n, dtype=np.float64)
    px, py = np.meshgrid(k * x, k * x, indexing="xy")  # py varies along rows (y), px along x
    drho = (u0 * u0) / (4 * cs2) * (np.cos(2 * px) + np.cos(2 * py))
    rho = (1.0 - drho).ravel()
    u = np.stack([-u0 * np.cos(px) * np.sin(py), u0 * np.sin(px) * np.cos(py)]).reshape(2, -1)
    f = O.init_equilibrium("D2Q9", rho, u, n, n, 1)

    def ke(pops):
        r, v = O.macro_fields(pops, "D2Q9", n, n, 1)
        return math.fsum(0.5 * r * (v ** 2).sum(0))

    e0 = ke(f)
    g = O.step(f, "D2Q9", op, n, n, 1, 1 / tau, steps=steps)
    assert abs(ke(g) - e0 * math.exp(-4 * nu * k * k * steps)) <= 1e-5


def _uniform(lat, nx, ny, conc_or_rho, ux=0.0, uy=0.0):
    n = nx * ny
    return O.init_equilibrium(lat, np.full(n, conc_or_rho), np.stack([np.full(n, ux), np.full(n, uy)]),
                              nx, ny, 1)


def test_reaction_kinetics_batch():
    """ReactionKineticsBatch (test_validation.cpp:1655-1702): C(t) = C0 / (1 + C0 k t)."""
    nx = ny = 16
    steps, k, tau_c = 200, 0.005, 0.8
    fluid = _uniform("D2Q9", nx, ny, 1.0)
    a = _uniform("D2Q5", nx, ny, 1.0)
    b = _uniform("D2Q5", nx, ny, 1.0)
    a2, b2 = O.reaction_ab(a, b, fluid, "D2Q9", nx, ny, 1, 1 / tau_c, k, steps=steps)
    want = 1.0 / (1.0 + k * steps)
    assert abs(a2[:, 0].sum() - want) <= 1e-4
    assert abs(b2[:, 0].sum() - want) <= 1e-4


def test_segregated_reactive_mixing():
    """SegregatedReactiveMixingD2Q5Cpu (test_validation.cpp:1712-1760)."""
    nx = ny = 32
    k, tau_c = 0.05, 0.8
    fluid = _uniform("D2Q9", nx, ny, 1.0)
    x = np.tile(np.arange(nx), ny)
    ca = np.where(x < nx // 2, 1.0, 0.0)
    a = O.init_equilibrium("D2Q5", ca, np.zeros((2, nx * ny)), nx, ny, 1)
    b = O.init_equilibrium("D2Q5", 1.0 - ca, np.zeros((2, nx * ny)), nx, ny, 1)
    m_a0, m_b0 = a.sum(), b.sum()
    a2, b2 = O.reaction_ab(a, b, fluid, "D2Q9", nx, ny, 1, 1 / tau_c, k, steps=20)
    ma, mb = a2.sum(), b2.sum()
    assert ma < m_a0 and mb < m_b0
    assert abs(ma - mb) <= 1e-10
    c_a, c_b = a2.sum(0), b2.sum(0)
    assert np.all(np.isfinite(c_a)) and np.all(np.isfinite(c_b))
    assert c_a.min() >= -1e-12 and c_b.min() >= -1e-12


def test_passive_scalar_advection_diffusion():
    """PassiveScalarAdvectionDiffusion (test_validation.cpp:1590-1646)."""
    nx, ny, steps, ux = 64, 8, 200, 0.05
    tau_c, c0, amp = 0.8, 1.0, 0.1
    D = (1.0 / 3.0) * (tau_c - 0.5)
    k = 2 * math.pi / nx
    fluid = _uniform("D2Q9", nx, ny, 1.0, ux, 0.0)
    x = np.tile(np.arange(nx, dtype=np.float64), ny)
    g = O.init_equilibrium("D2Q5", c0 + amp * np.sin(k * x),
                           np.stack([np.full(nx * ny, ux), np.zeros(nx * ny)]), nx, ny, 1)
    for _ in range(steps):  # the test steps the fluid (BGK, omega 1) and the scalar alternately
        fluid = O.step(fluid, "D2Q9", "BGK", nx, ny, 1, 1.0)
        g = O.scalar_step(g, fluid, "D2Q9", nx, ny, 1, 1 / tau_c, 0.0)
    want = c0 + amp * np.sin(k * (x - ux * steps)) * math.exp(-D * k * k * steps)
    assert np.max(np.abs(g.sum(0) - want)) <= 1e-4


def test_reaction_source_branches():
    """compute_reaction_ab_source (lattice_physics.hpp:712-743): equal-species
    branch A/(1+kA) and the exponential branch conserve B - A."""
    k = 0.3
    s = O.ORACLE.__getattr__  # noqa: F841 (binding check)
    import ctypes as C

    lib = C.CDLL(O.ORACLE_SO)
    lib.oracle_reaction_source_f64.restype = C.c_double
    lib.oracle_reaction_source_f64.argtypes = [C.c_double] * 3
    a = 0.7
    assert math.isclose(lib.oracle_reaction_source_f64(a, a, k), a / (1 + k * a) - a, rel_tol=1e-15)
    a, b = 0.9, 0.2
    src = lib.oracle_reaction_source_f64(a, b, k)
    # exact one-step solution of dA/dt = -k A B with B - A invariant
    d = b - a
    want = a * d * math.exp(-k * d) / (b - a * math.exp(-k * d)) - a
    assert math.isclose(src, want, rel_tol=1e-14)


# --- bitwise agreement with the reference's own build -----------------------
@needs_ref
@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("dtype", DTYPES, ids=["float", "double"])
def test_step_bitwise_vs_reference(lat, op, dtype):
    nx, ny, nz = SMALL[lat]
    f = U.random_state(lat, nx, ny, nz, dtype, seed=11)
    a = O.step(f, lat, op, nx, ny, nz, 1 / 0.6, steps=4)
    b = O.step(f, lat, op, nx, ny, nz, 1 / 0.6, steps=4, lib=O.REF)
    assert U.same_bits(a, b)


@needs_ref
@pytest.mark.parametrize("lat", LATS)
@pytest.mark.parametrize("dtype", DTYPES, ids=["float", "double"])
def test_adr_bitwise_vs_reference(lat, dtype):
    nx, ny, nz = SMALL[lat]
    sl = O.SCALAR_OF[lat]
    f = U.random_state(lat, nx, ny, nz, dtype, seed=12)
    a = U.random_scalar(sl, nx, ny, nz, dtype, seed=13)
    b = U.random_scalar(sl, nx, ny, nz, dtype, seed=14)
    assert U.same_bits(O.scalar_step(a, f, lat, nx, ny, nz, 1.2, 1e-3, steps=3),
                          O.scalar_step(a, f, lat, nx, ny, nz, 1.2, 1e-3, steps=3, lib=O.REF))
    r1 = O.reaction_ab(a, b, f, lat, nx, ny, nz, 1.2, 0.07, steps=3)
    r2 = O.reaction_ab(a, b, f, lat, nx, ny, nz, 1.2, 0.07, steps=3, lib=O.REF)
    assert all(U.same_bits(x, y) for x, y in zip(r1, r2))
    c1 = O.coupled_reaction(f, a, b, lat, "TRT", nx, ny, nz, 1 / 0.6, 1.2, 0.07, steps=3)
    c2 = O.coupled_reaction(f, a, b, lat, "TRT", nx, ny, nz, 1 / 0.6, 1.2, 0.07, steps=3, lib=O.REF)
    assert all(U.same_bits(x, y) for x, y in zip(c1, c2))
    assert U.same_bits(O.reactive_stats(a, b, sl, nx, ny, nz, 0.07),
                          O.reactive_stats(a, b, sl, nx, ny, nz, 0.07, lib=O.REF))


@needs_ref
@pytest.mark.parametrize("lat,q", [("D2Q9", 9), ("D3Q19", 19), ("D3Q27", 27)])
def test_mrt_transforms_bitwise_vs_reference(lat, q):
    f = np.random.default_rng(q).standard_normal(q)
    m = O.mrt_moments(lat, f)
    assert U.same_bits(m, O.mrt_moments(lat, f, lib=O.REF))
    assert U.same_bits(O.mrt_populations(lat, m), O.mrt_populations(lat, m, lib=O.REF))


@needs_ref
@pytest.mark.parametrize("lat", ["D2Q9", "D3Q19", "D3Q27", "D2Q5", "D3Q7"])
@pytest.mark.parametrize("dtype", DTYPES, ids=["float", "double"])
def test_equilibrium_bitwise_vs_reference(lat, dtype):
    u = [0.031, -0.017, 0.009][: O.D_OF[lat]]
    assert U.same_bits(O.equilibrium(lat, 1.013, u, dtype), O.equilibrium(lat, 1.013, u, dtype, lib=O.REF))
