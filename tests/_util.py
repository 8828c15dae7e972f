"""Shared helpers for the tests: seeded synthetic states and comparisons."""
import numpy as np

import oracle

Q_OF, D_OF = oracle.Q_OF, oracle.D_OF


def cells(lattice, nx, ny, nz):
    return nx * ny * (nz if D_OF[lattice] == 3 else 1)


def random_state(lattice, nx, ny, nz, dtype, seed, u_amp=0.03, rho_amp=0.02, neq=1e-3):
    """Equilibrium of a random density/velocity field plus a random
    non-equilibrium part, so every moment of the collision is exercised."""
    rng = np.random.default_rng(seed)
    n = cells(lattice, nx, ny, nz)
    rho = 1.0 + rho_amp * rng.standard_normal(n)
    u = u_amp * rng.standard_normal((D_OF[lattice], n))
    f = oracle.init_equilibrium(lattice, rho, u, nx, ny, nz, dtype)
    f += (neq * rng.standard_normal(f.shape)).astype(dtype)
    return f


def random_scalar(lattice, nx, ny, nz, dtype, seed, lo=0.0, hi=1.0):
    rng = np.random.default_rng(seed)
    n = cells(lattice, nx, ny, nz)
    c = rng.uniform(lo, hi, n)
    u = 0.02 * rng.standard_normal((D_OF[lattice], n))
    return oracle.init_equilibrium(lattice, c, u, nx, ny, nz, dtype)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def same_bits(got, want):
    """Bit-for-bit equality of two float arrays of one dtype, NaN payloads
    aside: NaN exactly where the other has NaN, every other element the same
    bit pattern (so +0 and -0 differ, unlike ==)."""
    got, want = np.asarray(got), np.asarray(want)
    if got.shape != want.shape or got.dtype != want.dtype:
        return False
    gn, wn = np.isnan(got), np.isnan(want)
    if not np.array_equal(gn, wn):
        return False
    as_int = {2: np.uint16, 4: np.uint32, 8: np.uint64}[got.dtype.itemsize]
    return np.array_equal(got.view(as_int)[~gn], want.view(as_int)[~wn])
