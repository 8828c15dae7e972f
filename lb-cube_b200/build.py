"""Builds the engine's shared library, lb-cube_b200/liblbcube_b200.so, in place.

Every CUDA translation unit under csrc/ is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) in parallel (host-only .cpp units
go through nvcc to the host compiler), then linked into one
library that exports the C ABI declared in include/lbcube_b200.h. Collision
code is built with ``--fmad=false`` so that multiply-adds are rounded exactly
as LB-Cube's CPU path rounds them (no contraction into FMA); that is what makes
the engine's steps bit-identical to the reference.

Usage: python lb-cube_b200/build.py [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblbcube_b200.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off"]
# Per-unit extra flags: exact (non-contracted) arithmetic for everything that
# must reproduce the reference's rounding.
UNITS = {
    "fluid_step.cu": ["--fmad=false"],
    "adr.cu": ["--fmad=false"],
    "stats.cu": ["--fmad=false"],
    "init.cu": ["--fmad=false"],
    "diag.cu": ["--fmad=false"],
    "macro.cu": ["--fmad=false"],
    "slab.cu": ["--fmad=false"],
    # the reaction source cancels near C_A = C_B: round it as the FP32 step does
    "adr_shifted.cu": ["--fmad=false"],
}


def _sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _obj(src):
    return os.path.join(BUILD, os.path.splitext(src)[0] + ".o")


def _headers():
    inc = os.path.join(os.path.dirname(HERE), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith((".h", ".cuh"))]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = _obj(src)
    extra = os.environ.get("LBCUBE_NVCC_FLAGS", "").split()  # e.g. -D overrides of tuning constants
    cmd = [NVCC, *COMMON, *ARCH, *UNITS.get(src, []), *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    return obj, (res.stdout + res.stderr)


DRIVERS = os.path.join(HERE, "drivers")
BIN = os.path.join(HERE, "bin")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))


def build_drivers(force: bool = False) -> list:
    """The ports of the reference's two drivers (drivers/*.cpp): host C++23
    executables on the C ABI, linked to the library next to them (bin/)."""
    os.makedirs(BIN, exist_ok=True)
    cxx = os.environ.get("CXX", shutil.which("g++") or "g++")
    inc = os.path.join(os.path.dirname(HERE), "include")
    out = []
    for name in ("lbm_sim", "lbm_reaction_sim"):
        src = os.path.join(DRIVERS, name + ".cpp")
        exe = os.path.join(BIN, name)
        deps = [src, os.path.join(DRIVERS, "driver_common.hpp"), os.path.join(inc, "lbcube_b200.h"), LIB]
        if force or _stale(exe, deps):
            cmd = [cxx, "-std=c++23", "-O2", "-ffp-contract=off", "-Wall", "-Wextra", f"-I{inc}",
                   f"-I{os.path.join(CUDA_HOME, 'include')}", src, "-o", exe, f"-L{HERE}", "-llbcube_b200",
                   "-Wl,-rpath,$ORIGIN/..", f"-L{os.path.join(CUDA_HOME, 'lib64')}", "-lcudart",
                   f"-Wl,-rpath,{os.path.join(CUDA_HOME, 'lib64')}"]
            res = subprocess.run(cmd, capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"driver build failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        out.append(exe)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile (if stale) and link the engine library; returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    headers = _headers()
    todo, objs = [], []
    for src in _sources():
        obj = _obj(src)
        objs.append(obj)
        if force or _stale(obj, [os.path.join(CSRC, src), *headers, __file__]):
            todo.append(src)
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            for obj, log in ex.map(lambda s: _compile(s, verbose), todo):
                if verbose and log.strip():
                    print(log)
    if force or todo or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    build_drivers(force)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)
