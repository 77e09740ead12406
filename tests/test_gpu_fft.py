"""Device mesh transforms vs numpy (FFTW conventions, unnormalised)."""
import numpy as np
import pytest

from oracle import restate as R

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [16, 32, 48, 96, 144, 192])
def test_r2c_matches_numpy(gpu_lib, n):
    from cola_halo_b200 import fft_r2c
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    got = fft_r2c(x).astype(np.complex128)
    want = np.fft.rfftn(x.astype(np.float64))
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 2e-6, err


@pytest.mark.parametrize("n", [16, 32, 48, 96, 144, 192])
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


@pytest.mark.parametrize("n", [384, 768])
def test_r2c_c2r_match_cufft_at_workload_sizes(gpu_lib, n):
    """The mesh transforms of the 128^3 and 256^3 workloads against cuFFT
    (torch.fft, float32, the same unnormalised conventions): both float32
    FFTs agree to float rounding, ~1e-6 of the spectrum's largest mode."""
    import torch
    from cola_halo_b200 import fft_c2r, fft_r2c
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n), dtype=np.float32)
    got = fft_r2c(x)
    xd = torch.from_numpy(x).cuda()
    want = torch.fft.rfftn(xd).cpu().numpy()
    del xd
    scale = np.abs(want).max()
    err = np.abs(got - want)
    assert err.max() / scale < 1e-5, err.max() / scale
    assert np.sqrt(np.mean(err.astype(np.float64) ** 2)) / scale < 1e-6
    back = fft_c2r(got)
    sd = torch.from_numpy(got).cuda()
    want_back = torch.fft.irfftn(sd, s=(n, n, n)).cpu().numpy() * float(n) ** 3
    del sd
    torch.cuda.empty_cache()
    scale_b = np.abs(want_back).max()
    err_b = np.abs(back - want_back)
    assert err_b.max() / scale_b < 1e-5, err_b.max() / scale_b
    np.testing.assert_allclose(back / float(n) ** 3, x, rtol=0, atol=1e-4)
