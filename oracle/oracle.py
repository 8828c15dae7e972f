"""Test infrastructure: numpy front end of the CPU oracle.

Loads ``oracle/liboracle.so`` (the C restatement of LB-Cube's CPU path,
``lbm_oracle.c``) and, when it has been built, ``oracle/_ref/libref.so`` (the
reference's own CPU path compiled from its unmodified headers through
``ref_bridge.cpp``). Both expose the same calls, so every helper below takes a
``lib`` argument: ``ORACLE`` (default) or ``REF``.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module. The engine never does.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref.so")

LATTICES = {"D2Q9": 0, "D3Q19": 1, "D3Q27": 2, "D2Q5": 3, "D3Q7": 4}
Q_OF = {"D2Q9": 9, "D3Q19": 19, "D3Q27": 27, "D2Q5": 5, "D3Q7": 7}
D_OF = {"D2Q9": 2, "D3Q19": 3, "D3Q27": 3, "D2Q5": 2, "D3Q7": 3}
SCALAR_OF = {"D2Q9": "D2Q5", "D3Q19": "D3Q7", "D3Q27": "D3Q7"}
COLLISIONS = {"BGK": 0, "TRT": 1, "MRT": 2, "RLBM": 3}
PRECISIONS = {np.float32: 0, np.float64: 1}

_sz = C.c_size_t
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (always possible: plain C)."""
    subprocess.run(["make", "-C", HERE, "oracle"], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _bind(lib, prefix):
    sig = {
        "step": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_double, C.c_int]),
        "scalar_step": (C.c_int, [C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double, C.c_double, C.c_int]),
        "reaction_ab": (C.c_int, [C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double, C.c_double, C.c_int]),
        "coupled_reaction": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _sz, _sz, _sz, C.c_double, C.c_double, C.c_double, C.c_int]),
        "equilibrium": (C.c_int, [C.c_int, C.c_int, C.c_double, _dp, _vp]),
        "mrt_moments": (C.c_int, [C.c_int, _dp, _dp]),
        "mrt_populations": (C.c_int, [C.c_int, _dp, _dp]),
    }
    if prefix == "oracle_":
        sig["reactive_stats"] = (C.c_int, [C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_double, C.c_int, _dp])
        sig["fluid_diagnostics"] = (C.c_int, [C.c_int, C.c_int, _vp, _sz, _sz, _sz, _dp])
        sig["fluid_diagnostics64"] = (C.c_int, [C.c_int, C.c_int, _vp, _sz, _sz, _sz, C.c_double, _dp])
        sig["macro_fields"] = (C.c_int, [C.c_int, C.c_int, _vp, _sz, _sz, _sz, _dp, _dp])
        sig["init_equilibrium"] = (C.c_int, [C.c_int, C.c_int, _dp, _dp, _vp, _sz, _sz, _sz])
    else:
        sig["reactive_stats"] = (C.c_int, [C.c_int, C.c_int, _vp, _vp, _sz, _sz, _sz, C.c_double, _dp])
        sig["write_vtk"] = (C.c_int, [C.c_int, C.c_int, _vp, _sz, _sz, _sz, _sz])
    out = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
        out[name] = fn
    return out


class _Lib:
    def __init__(self, path, prefix):
        self.path = path
        self.prefix = prefix
        self._fns = None

    @property
    def available(self) -> bool:
        return os.path.exists(self.path)

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if self._fns is None:
            if not os.path.exists(self.path):
                if self.prefix == "oracle_":
                    build()
                else:
                    raise FileNotFoundError(f"{self.path} not built (make -C oracle ref)")
            self._fns = _bind(C.CDLL(self.path), self.prefix)
        return self._fns[name]


ORACLE = _Lib(ORACLE_SO, "oracle_")
REF = _Lib(REF_SO, "ref_")


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_vp)


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def _prec(dtype) -> int:
    return PRECISIONS[np.dtype(dtype).type]


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned {rc}")


def step(f, lattice, collision, nx, ny, nz, omega, steps=1, lib=ORACLE):
    """``steps`` pull collide-stream steps of population array ``f`` [Q,Z,Y,X]."""
    f = np.ascontiguousarray(f)
    out = np.empty_like(f)
    _check(lib.step(LATTICES[lattice], _prec(f.dtype), COLLISIONS[collision], _ptr(f), _ptr(out),
                    nx, ny, nz, float(omega), int(steps)), "step")
    return out


def scalar_step(g, fluid, fluid_lattice, nx, ny, nz, omega_c, source=0.0, steps=1, lib=ORACLE):
    g = np.ascontiguousarray(g)
    fluid = np.ascontiguousarray(fluid, dtype=g.dtype)
    out = np.empty_like(g)
    _check(lib.scalar_step(LATTICES[fluid_lattice], _prec(g.dtype), _ptr(g), _ptr(out), _ptr(fluid),
                           nx, ny, nz, float(omega_c), float(source), int(steps)), "scalar_step")
    return out


def reaction_ab(a, b, fluid, fluid_lattice, nx, ny, nz, omega_c, k, steps=1, lib=ORACLE):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    fluid = np.ascontiguousarray(fluid, dtype=a.dtype)
    ao, bo = np.empty_like(a), np.empty_like(b)
    _check(lib.reaction_ab(LATTICES[fluid_lattice], _prec(a.dtype), _ptr(a), _ptr(ao), _ptr(b), _ptr(bo),
                           _ptr(fluid), nx, ny, nz, float(omega_c), float(k), int(steps)), "reaction_ab")
    return ao, bo


def coupled_reaction(fluid, a, b, fluid_lattice, collision, nx, ny, nz, omega, omega_c, k, steps=1,
                     lib=ORACLE):
    fluid, a, b = (np.array(x, copy=True, order="C") for x in (fluid, a, b))
    _check(lib.coupled_reaction(LATTICES[fluid_lattice], _prec(fluid.dtype), COLLISIONS[collision],
                                _ptr(fluid), _ptr(a), _ptr(b), nx, ny, nz, float(omega), float(omega_c),
                                float(k), int(steps)), "coupled_reaction")
    return fluid, a, b


STATS_FIELDS = ("mean_A", "mean_B", "var_A", "var_B", "covariance", "segregation_intensity",
                "true_reaction_rate", "mixed_reaction_rate")


def reactive_stats(a, b, scalar_lattice, nx, ny, nz, k, accumulate_f64=False, lib=ORACLE):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b, dtype=a.dtype)
    out = np.zeros(8, np.float64)
    if lib is REF:
        _check(lib.reactive_stats(LATTICES[scalar_lattice], _prec(a.dtype), _ptr(a), _ptr(b), nx, ny, nz,
                                  float(k), _dptr(out)), "reactive_stats")
    else:
        _check(lib.reactive_stats(LATTICES[scalar_lattice], _prec(a.dtype), _ptr(a), _ptr(b), nx, ny, nz,
                                  float(k), int(bool(accumulate_f64)), _dptr(out)), "reactive_stats")
    return out


def fluid_diagnostics(f, lattice, nx, ny, nz):
    f = np.ascontiguousarray(f)
    out = np.zeros(3, np.float64)
    _check(ORACLE.fluid_diagnostics(LATTICES[lattice], _prec(f.dtype), _ptr(f), nx, ny, nz, _dptr(out)),
           "fluid_diagnostics")
    return out


def fluid_diagnostics64(f, lattice, nx, ny, nz, speed_limit=math.inf):
    """The engine's diagnostics (FP64 sums): mass, KE, max |u|, non-finite
    cells, crash flag."""
    f = np.ascontiguousarray(f)
    out = np.zeros(5, np.float64)
    _check(ORACLE.fluid_diagnostics64(LATTICES[lattice], _prec(f.dtype), _ptr(f), nx, ny, nz,
                                      float(speed_limit), _dptr(out)), "fluid_diagnostics64")
    return out


def macro_fields(f, lattice, nx, ny, nz):
    """Density [N] and velocity [D, N] (double) of populations ``f``."""
    f = np.ascontiguousarray(f)
    n = nx * ny * (nz if D_OF[lattice] == 3 else 1)
    rho = np.zeros(n, np.float64)
    u = np.zeros((D_OF[lattice], n), np.float64)
    _check(ORACLE.macro_fields(LATTICES[lattice], _prec(f.dtype), _ptr(f), nx, ny, nz, _dptr(rho), _dptr(u)),
           "macro_fields")
    return rho, u


def equilibrium(lattice, rho, u, dtype=np.float64, lib=ORACLE):
    uu = np.zeros(3, np.float64)
    uu[: len(u)] = u
    out = np.zeros(Q_OF[lattice], dtype)
    _check(lib.equilibrium(LATTICES[lattice], _prec(dtype), float(rho), _dptr(uu), _ptr(out)), "equilibrium")
    return out


def reference_vtk(f, lattice, nx, ny, nz, step, workdir):
    """The reference build's write_vtk output for populations ``f`` (text), run
    in ``workdir`` (it writes lbm_<step, 6 digits>.vtk to the current directory)."""
    f = np.ascontiguousarray(f)
    old = os.getcwd()
    os.chdir(workdir)
    try:
        _check(REF.write_vtk(LATTICES[lattice], _prec(f.dtype), _ptr(f), nx, ny, nz, step), "write_vtk")
        with open(f"lbm_{step:06d}.vtk", "rb") as fh:
            return fh.read()
    finally:
        os.chdir(old)


def init_equilibrium(lattice, rho, u, nx, ny, nz, dtype=np.float64):
    """Equilibrium populations [Q, N] from rho [N] and u [D, N] (double inputs)."""
    rho = np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
    u = np.ascontiguousarray(u, dtype=np.float64).reshape(D_OF[lattice], -1)
    n = rho.size
    out = np.empty((Q_OF[lattice], n), dtype)
    _check(ORACLE.init_equilibrium(LATTICES[lattice], _prec(dtype), _dptr(rho), _dptr(u), _ptr(out),
                                   nx, ny, nz), "init_equilibrium")
    return out


def mrt_moments(lattice, f, lib=ORACLE):
    f = np.ascontiguousarray(f, dtype=np.float64)
    m = np.zeros_like(f)
    _check(lib.mrt_moments(LATTICES[lattice], _dptr(f), _dptr(m)), "mrt_moments")
    return m


def mrt_populations(lattice, m, lib=ORACLE):
    m = np.ascontiguousarray(m, dtype=np.float64)
    f = np.zeros_like(m)
    _check(lib.mrt_populations(LATTICES[lattice], _dptr(m), _dptr(f)), "mrt_populations")
    return f
