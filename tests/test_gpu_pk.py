"""Power spectrum estimator on the GPU vs the numpy estimator of the
oracle, on the CIC density of the same particles; plus the north-star
acceptance bar: the float32-atomic deposit's P(k) within 0.1 % of the oracle
(float64) deposit's up to the particle Nyquist wavenumber."""
import math

import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu
OM = 0.273


@pytest.mark.parametrize("deconv", [False, True])
def test_pk_matches_oracle(gpu_lib, bbks_table, deconv):
    from cola_halo_b200 import Simulation
    nc, factor, L = 32, 3, 200.0
    N = nc * factor
    p = lattice_particles(nc, L, 11, OM, 0.5, bbks_table)
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(p, 0.5, 0.5)
    sim.move()
    k, pk, modes = sim.power_spectrum(deconvolve_cic=deconv)
    x = R.wrap(p["x"], L)
    dens = R.cic_deposit(x, N, L, factor)
    ko, po, co = R.power_spectrum(dens, L, nbins=N // 2, deconvolve_cic=deconv)
    np.testing.assert_array_equal(modes, co)
    ok = co > 0
    np.testing.assert_allclose(k[ok], ko[ok], rtol=1e-12)
    # up to the particle Nyquist k = pi nc / L  <=> |n| <= nc/2
    upto = np.arange(1, N // 2 + 1) <= nc // 2
    rel = np.abs(pk[ok & upto] / po[ok & upto] - 1)
    assert rel.max() < 1e-3, rel.max()          # 0.1 %
    assert np.median(rel) < 1e-5


def test_pk_shot_noise_and_bins(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    nc, factor, L = 16, 2, 100.0
    p = lattice_particles(nc, L, 2, OM, 1.0, bbks_table)
    sim = Simulation(nc, nc * factor, L, OM)
    sim.set_particles(p, 1.0, 1.0)
    k1, p1, _ = sim.power_spectrum(nbins=8)
    k2, p2, _ = sim.power_spectrum(nbins=8, subtract_shot=True)
    # the two deposits differ only by float32 atomic ordering
    np.testing.assert_allclose(p1 - p2, L ** 3 / nc ** 3, rtol=0, atol=1e-6 * np.abs(p1).max())
    assert np.all(np.diff(k1) > 0) and abs(k1[0] - 2 * math.pi / L) < 0.5 * 2 * math.pi / L
