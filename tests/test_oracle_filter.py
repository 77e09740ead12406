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


def test_force_kernel_tables():
    """Reference values: the spectral, exact, uncorrected tables are the
    signed index, its square and 1; the difference operators approach the
    spectral gradient at small |n| and vanish at the Nyquist index."""
    N = 32
    g, lap, w = R.force_kernel_tables(N)
    s = np.where(np.arange(N) <= N // 2, np.arange(N), np.arange(N) - N)
    np.testing.assert_array_equal(g, s.astype(np.float32))
    np.testing.assert_array_equal(lap, (s * s).astype(np.float32))
    np.testing.assert_array_equal(w, np.ones(N, np.float32))
    g2, lap1, w2 = R.force_kernel_tables(N, 2, 1, 2)
    g4, _, w1 = R.force_kernel_tables(N, 4, 0, 1)
    assert abs(g2[1] - 1) < 1e-2 and abs(g4[1] - 1) < 1e-4        # O(w^2), O(w^4)
    assert abs(g2[N // 2]) < 1e-5 and abs(g4[N // 2]) < 1e-5
    assert abs(lap1[1] - 1) < 1e-2 and lap1[N // 2] == np.float32((N / np.pi) ** 2)
    # sinc^2(pi/2) = 4/pi^2 at the Nyquist index
    assert abs(w1[N // 2] - np.pi ** 2 / 4) < 1e-5 and abs(w2[N // 2] - np.pi ** 4 / 16) < 1e-4
    np.testing.assert_allclose(w2, w1 * w1, rtol=1e-6)


def test_force_kernel_reference_mode_is_the_reference():
    N = 16
    rng = np.random.default_rng(3)
    dk = rng.standard_normal((N, N, N // 2 + 1)) + 1j * rng.standard_normal((N, N, N // 2 + 1))
    for a in range(3):
        np.testing.assert_array_equal(R.force_spectrum(dk, N, 50.0, a, kernel=(0, 0, 0)),
                                      R.force_spectrum(dk, N, 50.0, a))
