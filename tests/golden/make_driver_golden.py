"""Generates tests/golden/drivers/: the outputs of LB-Cube's own drivers on their
CPU path, for the engine's ports of them (lb-cube_b200/drivers/).

The drivers are the reference's src/main.cpp (lbm_sim) and
src/simulate_reaction.cpp (lbm_reaction_sim), compiled unmodified by
lb-cube_b200/dropin.mk (which needs the reference tree: LBCUBE_REFERENCE or a
checkout next to this repository); their -cpu mode runs the reference's
step_cpu / step_reaction_AB and writes the files kept here. Regenerate with
    python tests/golden/make_driver_golden.py
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "drivers")
BIN = os.path.join(ROOT, "lb-cube_b200", "_build", "dropin")

# (executable, arguments, files kept)
RUNS = {
    "lbm_sim_tgv": ("lbm_sim", ["-nx", "12", "-ny", "10", "-nz", "8", "-steps", "40", "-out_freq", "20"],
                    ["diagnostics.csv", "lbm_000040.vtk"]),
    "lbm_sim_rest": ("lbm_sim", ["-nx", "8", "-ny", "6", "-nz", "4", "-steps", "10", "-out_freq", "5",
                                 "-init", "rest"], ["diagnostics.csv"]),
    "lbm_reaction_sim": ("lbm_reaction_sim", ["-nx", "32", "-ny", "24", "-steps", "60", "-out_freq", "20",
                                              "-k_react", "0.02"],
                         ["reaction_diagnostics.csv", "reaction_000060.vtk"]),
}


def main():
    ref = os.environ.get("LBCUBE_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
    subprocess.run(["make", "-f", os.path.join(ROOT, "lb-cube_b200", "dropin.mk"), f"REF={ref}"], check=True,
                   stdout=subprocess.DEVNULL)
    for name, (exe, args, keep) in RUNS.items():
        dst = os.path.join(OUT, name)
        os.makedirs(dst, exist_ok=True)
        with tempfile.TemporaryDirectory() as tmp:
            subprocess.run([os.path.join(BIN, exe), "-cpu", *args], cwd=tmp, check=True, stdout=subprocess.DEVNULL)
            for f in keep:
                shutil.copy(os.path.join(tmp, f), os.path.join(dst, f))
        with open(os.path.join(dst, "args.txt"), "w") as fh:
            fh.write(" ".join(args) + "\n")
        print(f"{name}: {', '.join(keep)}")


if __name__ == "__main__":
    sys.exit(main())
