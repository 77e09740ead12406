"""What the trained conv net gains: the learned-correction workload's
coarse run (128^3 particles on a 128^3 mesh, L = 300 Mpc/h, 10 steps from
z = 49) with the net's force correction against the same run without it,
both measured by the P(k) error up to half the particle Nyquist wavenumber
against the plain factor-3 (384^3) run on held-out seeds.  The net is
trained by the library's own forward and backward kernels on pairs made by
the method itself (factor-3 force minus coarse force along factor-3
trajectories)."""
import math

import numpy as np
import pytest

from cola_halo_b200.schedule import Schedule

pytestmark = pytest.mark.gpu
OM = 0.273


def test_net_lowers_pk_error(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.learned import (ConvNet, _final_positions, _lpt_particles, pk_error,
                                        power_spectrum_on, train_online)
    nc, L = 128, 300.0
    sched = Schedule.linear(0.02, 1.0, 10)
    fine = Simulation(nc, 3 * nc, L, OM)
    coarse = Simulation(nc, nc, L, OM)
    net = ConvNet(nc, seed=7)
    hist = train_online(net, coarse, fine, sched, list(range(1, 9)), bbks_table, lr=2e-3,
                        epochs=3)
    assert np.mean(hist[-10:]) < np.mean(hist[:10])
    kmax = 0.5 * math.pi * nc / L
    without, with_net = [], []
    for seed in (1001, 1002):
        p = _lpt_particles(nc, L, seed, OM, sched.a_init, bbks_table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        xf = _final_positions(fine, sched, fine.forces)
        coarse.set_particles(p, sched.a_init, sched.a_init)
        xc = _final_positions(coarse, sched, coarse.forces)
        coarse.set_particles(p, sched.a_init, sched.a_init)
        xl = _final_positions(coarse, sched, lambda: net.forces(coarse))
        k, pf, _ = power_spectrum_on(fine, xf, 1.0)
        _, pc, _ = power_spectrum_on(fine, xc, 1.0)
        _, pl, _ = power_spectrum_on(fine, xl, 1.0)
        without.append(pk_error(k, pc, pf, kmax))
        with_net.append(pk_error(k, pl, pf, kmax))
    print("\nP(k) error to 0.5 k_Nyq: coarse %.4f, coarse + net %.4f"
          % (np.mean(without), np.mean(with_net)))
    assert np.mean(with_net) < 0.9 * np.mean(without)
    for s in (fine, coarse):
        s.close()
    net.close()
