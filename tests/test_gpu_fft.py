"""Device mesh transforms vs numpy (FFTW conventions, unnormalised)."""
import numpy as np
import pytest

from oracle import restate as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [16, 32, 48, 96, 192])
def test_r2c_matches_numpy(gpu_lib, n):
    from cola_halo_b200 import fft_r2c
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    got = fft_r2c(x).astype(np.complex128)
    want = np.fft.rfftn(x.astype(np.float64))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 2e-6, err


@pytest.mark.parametrize("n", [16, 32, 48, 96, 192])
def test_c2r_non_hermitian_matches_fftw_convention(gpu_lib, n):
    """Random (non-Hermitian) half spectra: c2c over x, y then a z c2r that
    ignores Im of kz = 0 and kz = n/2 (pm.c:325-353 relies on this)."""
    from cola_halo_b200 import fft_c2r
    rng = np.random.default_rng(1000 + n)
    h = (rng.standard_normal((n, n, n // 2 + 1))
         + 1j * rng.standard_normal((n, n, n // 2 + 1))).astype(np.complex64)
    got = fft_c2r(h).astype(np.float64)
    want = R.c2r(h, n)
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 2e-6, err


def test_roundtrip(gpu_lib):
    from cola_halo_b200 import fft_c2r, fft_r2c
    n = 64
    rng = np.random.default_rng(7)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    back = fft_c2r(fft_r2c(x)) / n ** 3
    assert np.abs(back - x).max() < 1e-5
