"""CPU: the short form of the float reaction source's exp (rexp<float> in
lb-cube_b200/csrc/collide.cuh). For |x| < 2^-8 the device evaluates the Taylor
polynomial of degree 5 in double and rounds it to float; this checks, on a
million seeded arguments spread over that interval (and its edges), that the
rounded value equals float(exp(x)) computed in double, and that the double
value is within 2 units in the last place of exp(x). (numpy has no fused
multiply-add, so the polynomial here rounds twice per step: a weaker form than
the device's, which must pass all the more.)"""
import numpy as np


def _taylor5(d):
    p = d * (1.0 / 120.0) + 1.0 / 24.0
    p = p * d + 1.0 / 6.0
    p = p * d + 0.5
    p = p * d + 1.0
    return p * d + 1.0


def test_taylor_form_matches_exp_below_two_to_minus_8():
    rng = np.random.default_rng(0x5EED_E1)
    lim = 2.0 ** -8
    x = np.concatenate([rng.uniform(-lim, lim, 1_000_000), [-lim * (1 - 2 ** -24), lim * (1 - 2 ** -24), 0.0,
                                                            2.0 ** -30, -(2.0 ** -30)]])
    x = x.astype(np.float32).astype(np.float64)
    got = _taylor5(x)
    want = np.exp(x)
    ulp = np.spacing(want)
    assert np.max(np.abs(got - want) / ulp) <= 2.0
    assert np.array_equal(got.astype(np.float32), want.astype(np.float32))
