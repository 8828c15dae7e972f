"""CPU: LB-Cube's own drivers compile and link unchanged against the drop-in
header include/lattice_cuda.cuh and the engine library (needs the reference
sources, so it is skipped where they are absent)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# LB-Cube's source tree: LBCUBE_REFERENCE, else a checkout next to this repository
REF = os.environ.get("LBCUBE_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "src", "main.cpp")), reason="reference sources absent")
def test_reference_drivers_build_against_engine():
    import lbcube

    if not os.path.exists(lbcube.LIB_PATH):
        import build

        build.build()
    res = subprocess.run(["make", "-f", os.path.join(ROOT, "lb-cube_b200", "dropin.mk"), f"REF={REF}"],
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr
    for exe in ("lbm_sim", "lbm_reaction_sim"):
        out = os.path.join(ROOT, "lb-cube_b200", "_build", "dropin", exe)
        assert os.path.exists(out)
        syms = subprocess.run(["nm", "-D", "--undefined-only", out], capture_output=True, text=True).stdout
        assert "lbm_launch_" in syms  # the launchers resolve into the engine library
