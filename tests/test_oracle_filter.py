"""The oracle's force transfer function (restate.filter_at): piecewise
linear in |n| between knots spread over 0..sqrt(3) N / 2."""
import math

import numpy as np

from oracle import restate as R


def test_filter_is_piecewise_linear():
    N, nk = 48, 11
    knots = np.random.default_rng(1).uniform(0.5, 1.5, nk).astype(np.float32)
    den = np.arange(0, 3 * (N // 2) ** 2 + 1)
    got = R.filter_at(den, knots, N)
    r = np.sqrt(den) * (nk - 1) / (math.sqrt(3.0) * N / 2)
    want = np.interp(r, np.arange(nk), knots.astype(np.float64))
    assert np.abs(got - want).max() < 1e-6
    # exact at the knots that fall on integer |n|^2
    assert got[0] == knots[0]


def test_unit_filter_leaves_the_force_unchanged():
    N = 16
    rng = np.random.default_rng(2)
    dk = rng.standard_normal((N, N, N // 2 + 1)) + 1j * rng.standard_normal((N, N, N // 2 + 1))
    for a in range(3):
        np.testing.assert_array_equal(R.force_spectrum(dk, N, 50.0, a, np.ones(5)),
                                      R.force_spectrum(dk, N, 50.0, a))
