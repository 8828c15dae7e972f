"""CPU: the division-free FP32 quotients x / 3 and x / 6 of the D3Q27 MRT
population transform (div_exact_const, lb-cube_b200/csrc/collide.cuh) equal
IEEE division wherever the transform uses them.

The transform takes the fast path only when every dividend is finite and, for
a division by 6, zero or at least 2^-124 in magnitude; it never depends on the
sign of a zero quotient. So the claim to prove is: for every finite nonzero x
(D = 3), resp. every x with |x| >= 2^-124 (D = 6), the quotient is the IEEE
one. The helper (div_const_check.c, the same three IEEE operations on the
host) checks every FP32 pattern with |x| < 2^-98 (all subnormals and the
binades where intermediate values can underflow), the binade [1, 2) and the
top binade. For 2^-98 <= |x| < 2^127 every rounded value (q0, r, q) is a
normal number (r is zero or a multiple of 2^-125), so all three operations
commute with scaling by a power of two and [1, 2) stands for every binade in
between.

FP64 rests on Markstein's theorem (RN(1/D) is within half an ulp of 1/D and
RN(x RN(1/D)) within one ulp of x / D, so the corrected quotient is the
correctly rounded one away from underflow and overflow); the FP64 transform
keeps every dividend at 0 or >= 2^-960. The test samples 5e7 random bit
patterns over all exponents and 5e7 dividends whose quotient lies next to a
rounding midpoint, per divisor.
"""
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))

RANGES = [(0x00000000, 0x0E7FFFFF),   # |x| < 2^-98, including zero and subnormals
          (0x3F800000, 0x3FFFFFFF),   # [1, 2)
          (0x7F000000, 0x7F800000)]   # top binade and infinity


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("divc") / "div_const_check")
    subprocess.run(["gcc", "-O3", "-fopenmp", "-mfma", "-ffp-contract=off", os.path.join(HERE, "div_const_check.c"),
                    "-o", exe, "-lm"], check=True)
    return exe


@pytest.mark.parametrize("d", [3, 6])
def test_div_exact_const_matches_ieee(checker, d):
    bad_total = 0
    for lo, hi in RANGES:
        out = subprocess.run([checker, str(d), f"{lo:x}", f"{hi:x}"], check=True, capture_output=True,
                             text=True).stdout.split()
        n, bad, bad_range, worst = int(out[0]), int(out[1]), int(out[2]), float.fromhex(out[3])
        assert n == 2 * (hi - lo + 1)
        assert bad_range == 0, f"D={d}: {bad_range} mismatches at |x| >= 2^-124 in [{lo:#x}, {hi:#x}]"
        if d == 3:
            # only -0 (gives +0) and +-inf (gives NaN) differ
            assert worst == 0.0
        else:
            assert worst <= 2.0 ** -125
        bad_total += bad
    # D = 3: -0 and +-inf; D = 6: -0, +-inf and the near-subnormal dividends
    assert bad_total == 3 if d == 3 else bad_total > 3


@pytest.mark.parametrize("d", [3, 6])
def test_div_exact_const_f64_samples(checker, d):
    out = subprocess.run([checker, str(d), "f64", "50000000", str(d)], check=True, capture_output=True,
                         text=True).stdout.split()
    assert int(out[0]) == 100000000
    assert int(out[1]) == 0, f"D={d}: {out[1]} FP64 mismatches"
