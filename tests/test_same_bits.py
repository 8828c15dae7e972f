"""The bit-equality check that the parity tests use: it tells +0 from -0,
accepts NaN only where the other array has NaN, and rejects a dtype change."""
import numpy as np

import _util as U


def test_same_bits():
    for dt in (np.float32, np.float64):
        a = np.array([0.0, np.nan, 1.5, -np.inf], dt)
        assert U.same_bits(a, a.copy())
        assert not U.same_bits(a, np.array([-0.0, np.nan, 1.5, -np.inf], dt))
        assert not U.same_bits(a, np.array([0.0, 0.0, 1.5, -np.inf], dt))
        assert not U.same_bits(a, np.array([0.0, np.nan, np.nextafter(dt(1.5), dt(2)), -np.inf], dt))
        assert not U.same_bits(a, a.astype(np.float64 if dt is np.float32 else np.float32))
        assert not U.same_bits(a, a[:3])
