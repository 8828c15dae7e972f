"""GPU: the engine's ports of LB-Cube's two drivers against the drivers' own
CPU-path output.

lb-cube_b200/bin/lbm_sim and lbm_reaction_sim (sources in
lb-cube_b200/drivers/) take the reference drivers' command line and write the
same files, with the statistics reduced on the device and kernel-only timing.
The fixtures in tests/golden/drivers/ are what the reference's unmodified
drivers write with -cpu for the same arguments
(tests/golden/make_driver_golden.py).
* lbm_sim: the step, mass, kinetic-energy and max-|u| columns of
  diagnostics.csv agree to 1e-12 relative (the engine adds the FP64 terms in
  another order; max |u| is exact); the VTK file is byte-identical.
* lbm_reaction_sim: the nine-column statistics agree to 1e-12 relative (the
  reaction's exp() may differ in the last bit, and the sums are ordered
  differently); every number of the VTK file agrees to 1e-12 relative.
* both report a kernel-only MLUPS figure.
"""
import csv
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "lb-cube_b200", "bin")
GOLD = os.path.join(ROOT, "tests", "golden", "drivers")


@pytest.fixture(scope="module")
def ports(engine):
    import build

    return build.build_drivers()


def _run(tmp_path, exe, case):
    args = open(os.path.join(GOLD, case, "args.txt")).read().split()
    res = subprocess.run([os.path.join(BIN, exe), "-gpu", *args], cwd=tmp_path, capture_output=True, text=True,
                         timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "Kernel performance:" in res.stdout
    return res.stdout


def _close(a, b, rel=1e-12):
    return abs(a - b) <= rel * max(abs(a), abs(b), 1e-300)


def _compare_csv(got_path, want_path):
    got = list(csv.reader(open(got_path)))
    want = list(csv.reader(open(want_path)))
    assert got[0] == want[0] and len(got) == len(want)
    for g, w in zip(got[1:], want[1:]):
        assert g[0] == w[0]
        for x, y in zip(map(float, g[1:]), map(float, w[1:])):
            assert _close(x, y), (g, w)


@pytest.mark.parametrize("case", ["lbm_sim_tgv", "lbm_sim_rest"])
def test_lbm_sim_port(ports, tmp_path, case):
    _run(tmp_path, "lbm_sim", case)
    _compare_csv(tmp_path / "diagnostics.csv", os.path.join(GOLD, case, "diagnostics.csv"))
    for name in os.listdir(os.path.join(GOLD, case)):
        if name.endswith(".vtk"):
            assert (tmp_path / name).read_bytes() == open(os.path.join(GOLD, case, name), "rb").read(), name


def test_lbm_reaction_sim_port(ports, tmp_path):
    case = "lbm_reaction_sim"
    _run(tmp_path, "lbm_reaction_sim", case)
    _compare_csv(tmp_path / "reaction_diagnostics.csv", os.path.join(GOLD, case, "reaction_diagnostics.csv"))
    got = open(tmp_path / "reaction_000060.vtk").read().split("\n")
    want = open(os.path.join(GOLD, case, "reaction_000060.vtk")).read().split("\n")
    assert len(got) == len(want)
    for g, w in zip(got, want):
        if g == w:
            continue
        gv, wv = g.split(), w.split()
        assert len(gv) == len(wv), (g, w)
        for x, y in zip(gv, wv):
            assert _close(float(x), float(y)), (g, w)


def test_ports_reject_the_cpu_path(ports, tmp_path):
    res = subprocess.run([os.path.join(BIN, "lbm_sim"), "-cpu"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=60)
    assert res.returncode != 0 and "GPU only" in res.stderr
