"""Batched realizations (uneven boxes and step counts, one graph launch) vs
the single-realization path on the same initial particles: positions and
per-realization P(k)."""
import numpy as np
import pytest

from cola_halo_b200.schedule import Schedule
from tests.helpers import lattice_particles, periodic_diff

pytestmark = pytest.mark.gpu
OM = 0.273


def test_batch_matches_single_runs(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.batch import Batch
    rng = np.random.default_rng(42)
    specs, ics = [], []
    for i in range(5):
        nc = 16 if i % 2 else 32
        L = float(rng.uniform(100, 200))
        nsteps = int(rng.integers(3, 9))
        specs.append(dict(nc=nc, ngrid=3 * nc, boxsize=L, a_init=0.02, nsteps=nsteps, aout=1.0))
        ics.append(lattice_particles(nc, L, 200 + i, OM, 0.02, bbks_table))
    b = Batch(specs, OM, nstreams=3)
    for i, p in enumerate(ics):
        b.set_particles(i, p)
    b.run()
    assert b.num_nodes() > 10 * len(specs)
    first = [b.snapshot(i) for i in range(len(specs))]
    b.run()                      # relaunch restarts from the stored particles
    for i, s in enumerate(specs):
        again = b.snapshot(i)
        L = s["boxsize"]
        assert periodic_diff(again["x"], first[i]["x"], L).max() <= 1e-5 * L
        sim = Simulation(s["nc"], s["ngrid"], L, OM)
        sim.set_particles(ics[i], 0.02, 0.02)
        snaps = sim.run(Schedule.linear(0.02, 1.0, s["nsteps"]), zout=(0.0,))
        ref = snaps[-1][1]
        assert periodic_diff(first[i]["x"], ref["x"], L).max() <= 1e-5 * L
        np.testing.assert_array_equal(first[i]["id"], ref["id"])
        k, p, m = b.power_spectrum(i)
        ks, ps, ms = sim.power_spectrum()
        np.testing.assert_array_equal(m, ms)
        ok = m > 0
        assert np.abs(p[ok] / ps[ok] - 1).max() < 1e-3
        sim.close()
    b.close()


def _close_enough(got, ref, L):
    """Positions of two float-atomic runs of the same realization: the bar
    of the one-GPU workload's parity test (all but 1 in 10^5 particles
    within 1e-5 of the box, none beyond 5e-5)."""
    d = periodic_diff(got["x"], ref["x"], L).max(axis=1) / L
    return (d > 1e-5).sum() <= len(d) // 100000 and d.max() <= 5e-5, d.max()


@pytest.mark.parametrize("sort_every", [0, 3])
def test_batch_at_batched_workload_sizes(gpu_lib, bbks_table, sort_every):
    """Realizations of the batched workload's shape (128^3 particles on 384^3
    meshes, L in 250-400 Mpc/h, 5-20 steps from z = 49) against the single
    run of each, with the cell-order sort inside the graph (every third
    move) and without it."""
    from cola_halo_b200 import Simulation
    from cola_halo_b200.batch import Batch
    rng = np.random.default_rng(7)
    specs, ics = [], []
    for i in range(3):
        L = float(rng.uniform(250, 400))
        nsteps = int(rng.integers(5, 21))
        specs.append(dict(nc=128, ngrid=384, boxsize=L, a_init=0.02, nsteps=nsteps, aout=1.0))
        ics.append(lattice_particles(128, L, 300 + i, OM, 0.02, bbks_table))
    b = Batch(specs, OM, nstreams=2)
    b.set_sort_interval(sort_every)
    for i, p in enumerate(ics):
        b.set_particles(i, p)
    b.run()
    for i, s in enumerate(specs):
        L = s["boxsize"]
        got = b.snapshot(i)
        sim = Simulation(128, 384, L, OM)
        sim.set_sort_interval(sort_every)
        sim.set_particles(ics[i], 0.02, 0.02)
        ref = sim.run(Schedule.linear(0.02, 1.0, s["nsteps"]), zout=(0.0,))[-1][1]
        ok, dmax = _close_enough(got, ref, L)
        assert ok, (i, s, dmax)
        np.testing.assert_array_equal(got["id"], ref["id"])
        k, p, m = b.power_spectrum(i)
        ks, ps, ms = sim.power_spectrum()
        np.testing.assert_array_equal(m, ms)
        upto = (np.arange(1, len(m) + 1) <= 64) & (m > 0)   # to the particle Nyquist
        assert np.abs(p[upto] / ps[upto] - 1).max() < 1e-3
        sim.close()
    b.close()
