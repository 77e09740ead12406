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
