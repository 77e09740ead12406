"""cg_pk_bins_noalloc (shell sums from a fixed device array, no allocation)
against the allocating cg_sim_power_spectrum on the same particles, two
calls in a row.  Kept in its own file named to be collected last, so it runs
both alone and after every other test of the session."""
import numpy as np
import pytest

from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu
OM = 0.273


def _noalloc(lib, d_spec, n, L, nbins, flags, np_count):
    k = np.zeros(nbins)
    pk = np.zeros(nbins)
    m = np.zeros(nbins)
    rc = lib.cg_pk_bins_noalloc(d_spec, n, L, nbins, flags, k.ctypes.data, pk.ctypes.data,
                                m.ctypes.data, np_count, None)
    assert rc == 0, lib.cg_last_error()
    return k, pk, m


@pytest.mark.parametrize("flags", [0, 3])
def test_noalloc_matches_power_spectrum_twice(gpu_lib, bbks_table, flags):
    import torch
    from cola_halo_b200 import Simulation
    nc, factor, L = 32, 2, 150.0
    N = nc * factor
    nbins = N // 2
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(lattice_particles(nc, L, 21, OM, 0.5, bbks_table), 0.5, 0.5)
    sim.move()
    k0, p0, m0 = sim.power_spectrum(nbins, deconvolve_cic=bool(flags & 1),
                                     subtract_shot=bool(flags & 2))
    # the density mesh the call above binned, transformed by the library
    delta = np.zeros(N * N * N, dtype=np.float32)
    assert gpu_lib.cg_sim_get_mesh(sim.h, 0, delta.ctypes.data) == 0
    spec = np.zeros(N * N * (N // 2 + 1) * 2, dtype=np.float32)
    assert gpu_lib.cg_fft_r2c(N, delta.ctypes.data, spec.ctypes.data) == 0
    d_spec = torch.from_numpy(spec).cuda()
    torch.cuda.synchronize()
    for _ in range(2):
        k, pk, m = _noalloc(gpu_lib, d_spec.data_ptr(), N, L, nbins, flags, nc ** 3)
        np.testing.assert_array_equal(m, m0)
        np.testing.assert_allclose(k, k0, rtol=1e-12)
        # both spectra are float32 FFTs of the same mesh; the bins sum in double
        np.testing.assert_allclose(pk, p0, rtol=1e-5, atol=1e-6 * np.abs(p0).max())


def test_noalloc_rejects_more_bins_than_scratch(gpu_lib):
    import torch
    n = 16
    d_spec = torch.zeros(n * n * (n // 2 + 1) * 2, dtype=torch.float32, device="cuda")
    nb = 1024                       # CG_PK_NOALLOC_MAX_BINS in colagpu.h
    k = np.zeros(nb + 1)
    rc = gpu_lib.cg_pk_bins_noalloc(d_spec.data_ptr(), n, 100.0, nb + 1, 0, k.ctypes.data,
                                    k.ctypes.data, k.ctypes.data, 0, None)
    assert rc != 0
    assert b"1024" in gpu_lib.cg_last_error()
