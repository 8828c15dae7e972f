"""Seeded synthetic workloads with the shapes of LB-Cube's studies, built on the
host so that the CPU path and the engine start from the same bits.

Every field is made with integer arithmetic (splitmix64) and single IEEE
operations on 1-D tables of transcendental values; the tables themselves are
returned with the fields, so a check that must reproduce a field on another
machine can pass the stored tables back in instead of recomputing them with
that machine's libm.
"""
from __future__ import annotations

import math

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, count: int) -> np.ndarray:
    """The first `count` outputs of splitmix64 started at `seed` (Steele,
    Lea and Flood, "Fast splittable pseudorandom number generators", 2014):
    state_i = seed + i * 0x9E3779B97F4A7C15, then two xor-shift-multiply
    rounds and a final xor-shift. Plain uint64 arithmetic, modulo 2^64."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + np.arange(1, count + 1, dtype=np.uint64) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def uniform_pm1(seed: int, count: int) -> np.ndarray:
    """`count` doubles uniform on [-1, 1): the top 53 bits of splitmix64 scaled
    by 2^-52, minus 1 (every step exact)."""
    return (splitmix64(seed, count) >> np.uint64(11)).astype(np.float64) * 2.0 ** -52 - 1.0


SHEAR_SEED = 0x5EED_C3
SHEAR_U0 = 0.04
SHEAR_DELTA = 8.0


def shear_layer_tables(n: int, u0: float = SHEAR_U0, delta: float = SHEAR_DELTA) -> dict:
    """The 1-D tables of the double shear layer: u_x of each row
    y = j / n (u0 tanh((n / delta)(y - 1/4)) below y = 1/2, u0 tanh((n /
    delta)(3/4 - y)) above: the periodic double shear layer of
    src/turbulent_shear_layer.cpp:61-63 with a shear thickness of `delta`
    cells) and cos(2 pi x) of each column x = i / n, from the math module."""
    ux_row = np.array([u0 * math.tanh((n / delta) * (j / n - 0.25)) if j / n <= 0.5 else
                       u0 * math.tanh((n / delta) * (0.75 - j / n)) for j in range(n)], np.float64)
    cos_col = np.array([math.cos(2.0 * math.pi * (i / n)) for i in range(n)], np.float64)
    return {"ux_row": ux_row, "cos_col": cos_col}


def reactive_shear_layer(n: int = 1024, tau: float = 0.6, tables: dict | None = None,
                         seed: int = SHEAR_SEED, u0: float = SHEAR_U0, peclet: float = 1000.0,
                         damkohler: float = 1.0) -> dict:
    """The 2-D reactive-mixing workload: a D2Q9 fluid on an n x n periodic box
    with the double shear layer of `shear_layer_tables` plus a transverse
    perturbation u_y = u0 1e-3 (cos(2 pi x) + r), r uniform on [-1, 1) from
    splitmix64(seed), rho = 1; species A = 1 in the top half (y > 1/2) and
    B = 1 in the bottom half, as in src/turbulent_shear_layer.cpp:86-87.
    Transport and reaction follow from Pe = u0 L / D = `peclet` and
    Da = k C0 L / u0 = `damkohler` with L = n and C0 = 1; the D2Q5 diffusivity
    is D = (tau_c - 1/2) / 3.

    Returns FP32 fields (rho [n*n], u [2, n*n], a0 [n*n], b0 [n*n], row-major
    with x fastest) and the parameters."""
    t = tables if tables is not None else shear_layer_tables(n, u0)
    ux_row = np.asarray(t["ux_row"], np.float64)
    cos_col = np.asarray(t["cos_col"], np.float64)
    r = uniform_pm1(seed, n * n).reshape(n, n)
    ux = np.broadcast_to(ux_row[:, None], (n, n))
    uy = (u0 * 1e-3) * (cos_col[None, :] + r)
    u = np.stack([ux, uy]).astype(np.float32).reshape(2, n * n)
    rows = np.arange(n) / n
    top = np.broadcast_to((rows > 0.5)[:, None], (n, n)).reshape(-1)
    diffusivity = u0 * n / peclet
    return {"n": n, "tau": tau, "tau_c": 0.5 + 3.0 * diffusivity, "k": damkohler * u0 / n,
            "rho": np.ones(n * n, np.float32), "u": np.ascontiguousarray(u),
            "a0": top.astype(np.float32), "b0": (~top).astype(np.float32), "tables": t}
