"""GPU: LB-Cube's own drivers, unmodified, linked against the engine.

lbm_sim (src/main.cpp) and lbm_reaction_sim (src/simulate_reaction.cpp) are
compiled by lb-cube_b200/dropin.mk with include/lattice_cuda.cuh shadowing the
reference header. The same executable runs its CPU path (-cpu, the reference's
step_cpu) and its GPU path (-gpu, this engine through the launcher templates).
* lbm_sim: diagnostics CSV and VTK output are byte-identical.
* lbm_reaction_sim: fluid fields identical; the reaction's exp() may differ in
  the last bit, so the 9-column statistics agree to relative 1e-12.
The executables are built where the reference sources exist and travel with
the repository; the test is skipped when they are absent.
"""
import csv
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "lb-cube_b200", "_build", "dropin")


def _run(tmp_path, exe, mode, args):
    d = tmp_path / mode
    d.mkdir()
    res = subprocess.run([os.path.join(BIN, exe), f"-{mode}", *args], cwd=d, capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    return d


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "lbm_sim")), reason="drop-in build absent")
def test_lbm_sim_gpu_equals_cpu(tmp_path):
    args = ["-nx", "24", "-ny", "20", "-nz", "16", "-steps", "60", "-out_freq", "30"]
    c = _run(tmp_path, "lbm_sim", "cpu", args)
    g = _run(tmp_path, "lbm_sim", "gpu", args)
    for name in ("diagnostics.csv", "lbm_000030.vtk", "lbm_000060.vtk"):
        assert (c / name).read_bytes() == (g / name).read_bytes(), name


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "lbm_reaction_sim")), reason="drop-in build absent")
def test_lbm_reaction_sim_gpu_matches_cpu(tmp_path):
    args = ["-nx", "48", "-ny", "40", "-steps", "50", "-out_freq", "10", "-k_react", "0.02"]
    c = _run(tmp_path, "lbm_reaction_sim", "cpu", args)
    g = _run(tmp_path, "lbm_reaction_sim", "gpu", args)
    rc = list(csv.reader(open(c / "reaction_diagnostics.csv")))
    rg = list(csv.reader(open(g / "reaction_diagnostics.csv")))
    assert rc[0] == rg[0] and len(rc) == len(rg) == 7  # header, step 0, 5 outputs
    for a, b in zip(rc[1:], rg[1:]):
        assert a[0] == b[0]
        for x, y in zip(map(float, a[1:]), map(float, b[1:])):
            assert abs(x - y) <= 1e-12 * max(abs(x), 1e-9)
