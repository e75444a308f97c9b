"""Initial conditions of ch_swe_b200.testcases against the oracle's restatement of
the reference generators (test_fields_mod.f90)."""
import numpy as np

from oracle.oracle import Oracle


def test_gaussian_hill_matches_oracle(oracle_built):
    from ch_swe_b200 import testcases
    o = Oracle(24)
    a = testcases.gaussian_hill(24, 0.7, 0.3, 0.2, 1.5)
    b = o.gaussian(0.7, 0.3, 0.2, 1.5)
    for x, y in zip(a, b):
        assert np.abs(x - y).max() <= 1e-14


def test_williamson2_matches_oracle(oracle_built):
    from ch_swe_b200 import testcases
    axis = (0.3, 0.1, 0.9)
    o = Oracle(20, axis=axis)
    a = testcases.williamson2(20, u0=20.0, h_mean=3000.0, axis=axis, linear_mode=True)
    b = o.ts2(20.0, 3000.0, axis, True)
    for x, y in zip(a, b):
        assert np.abs(x - y).max() <= 1e-13 * np.abs(y).max()
