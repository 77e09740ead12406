"""The plain-COLA workloads end to end against the reference's own CPU code.

  64^3 particles on a 192^3 mesh, L = 200 Mpc/h (the CPU-runnable case)
  256^3 particles on a 768^3 mesh, L = 600 Mpc/h (the one-GPU case)

both with BBKS initial conditions at z = 49 and 10 COLA steps linear in a to
z = 0 (main.c:117-206 control flow).  Both paths start from the reference's
own 2LPT output: lpt_set_displacement of the reference (lpt.c:145-578, built
unchanged in oracle/_ref) generates the particles, which are handed to the
reference's pm.c / cola.c / move.c on the host and to this library on the
GPU.  The z = 0 snapshots (cola_set_snapshot, cola.c:341-416) must agree:

  * positions within 1e-5 of the box size: every particle at 64^3; at 256^3
    all but at most 1 particle in 10^5 (and none beyond 5e-5 of the box);
  * velocities within 1e-5 of the largest speed in rms;
  * P(k) of the GPU's float32-atomic deposit of its z = 0 positions within
    0.1 % of the oracle's float64 deposit (oracle/restate.py) of the
    reference's z = 0 positions, in every bin up to the particle Nyquist
    wavenumber pi nc / L.

Why not every particle at 256^3: the deposit adds float32 weights with
atomics, here and in the reference (pm.c:73-80, `omp atomic`), so neither
code reproduces itself bit for bit, and 10 steps amplify the rounding in the
densest halos.  Two GPU runs of the 256^3 workload that differ only in the
order of their atomic additions end up to 1.2e-5 of the box apart, with 1 to
a few particles beyond 1e-5; the GPU and the reference differ by at most
2e-5 with 17 of 16,777,216 beyond.  The test runs the GPU twice and prints
both comparisons.

The reference runs on the host's cores with the project's double-precision
shim FFT in place of FFTW (oracle/Makefile); the 256^3 case takes a few
minutes of host time.
"""
import numpy as np
import pytest

from cola_halo_b200.schedule import Schedule
from oracle import restate as R
from tests.helpers import periodic_diff
from tests.test_gpu_run import reference_run

pytestmark = pytest.mark.gpu
OM = 0.273


@pytest.mark.parametrize("nc,factor,L", [(64, 3, 200.0), (256, 3, 600.0)],
                         ids=["64p_192mesh", "256p_768mesh"])
def test_workload_matches_reference(gpu_lib, ref, bbks_table, nc, factor, L):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.types import PARTICLE_DTYPE
    N = nc * factor
    sched = Schedule.linear(0.02, 1.0, 10)          # z = 49 -> 0, 10 steps
    ics, snaps = reference_run(ref, bbks_table, nc, factor, L, 100, sched, zout=(0.0,))
    (a_r, s_r), = snaps
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(ics, sched.a_init, sched.a_init)
    (a_g, s_g), = sim.run(sched, zout=(0.0,), check_density=True)
    assert a_r == a_g == 1.0
    np.testing.assert_array_equal(s_g["id"], s_r["id"])

    dx = periodic_diff(s_g["x"], s_r["x"], L).max(axis=1) / L
    dv = s_g["v"].astype(np.float64) - s_r["v"]
    vmax = np.abs(s_r["v"]).max()
    n_out = int((dx > 1e-5).sum())
    print("\n%d^3/%d^3 GPU vs reference: max |dx|/L = %.2e (99.99%%: %.2e), %d of %d beyond "
          "1e-5; rms |dv|/vmax = %.2e, max |dv|/vmax = %.2e"
          % (nc, N, dx.max(), np.quantile(dx, 0.9999), n_out, nc ** 3,
             np.sqrt(np.mean(dv ** 2)) / vmax, np.abs(dv).max() / vmax))
    if nc <= 64:
        assert dx.max() <= 1e-5
    else:
        # the same run again: only the order of the float atomic additions
        # differs, which sets the floor any float32-atomic code meets
        sim2 = Simulation(nc, N, L, OM)
        sim2.set_particles(ics, sched.a_init, sched.a_init)
        (_, s_g2), = sim2.run(sched, zout=(0.0,))
        sim2.close()
        d2 = periodic_diff(s_g["x"], s_g2["x"], L).max(axis=1) / L
        print("GPU vs GPU (atomic order only): max |dx|/L = %.2e (99.99%%: %.2e), %d beyond 1e-5"
              % (d2.max(), np.quantile(d2, 0.9999), int((d2 > 1e-5).sum())))
        assert n_out <= nc ** 3 // 100000
        assert dx.max() <= 5e-5
    assert np.sqrt(np.mean(dv ** 2)) <= 1e-5 * vmax

    # P(k) of the z = 0 positions: the GPU estimator (float32 atomics) on the
    # GPU's particles against the oracle's float64 deposit of the reference's
    p = np.zeros(nc ** 3, dtype=PARTICLE_DTYPE)
    p["x"] = s_g["x"]
    sim.set_particles(p, 1.0, 1.0)
    sim.move()                                       # wrap (move.c:34-41)
    k, pk, modes = sim.power_spectrum(nbins=N // 2)
    sim.close()
    dens = R.cic_deposit(R.wrap(s_r["x"], L), N, L, factor)
    ko, po, co = R.power_spectrum(dens, L, nbins=N // 2)
    del dens
    np.testing.assert_array_equal(modes, co)
    upto = (np.arange(1, N // 2 + 1) <= nc // 2) & (co > 0)   # |n| <= nc/2: k <= pi nc / L
    rel = np.abs(pk[upto] / po[upto] - 1)
    print("P(k) to the particle Nyquist: max rel diff %.2e over %d bins" % (rel.max(), upto.sum()))
    assert rel.max() < 1e-3
