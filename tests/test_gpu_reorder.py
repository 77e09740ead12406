"""Cell order of the particle arrays (reorder.cu): the sort is internal, so
every output stays in the caller's order, bit for bit where no float sum
changes and within float rounding of the deposit otherwise."""
import numpy as np
import pytest

from cola_halo_b200.types import PARTICLE_DTYPE

pytestmark = pytest.mark.gpu
OM = 0.273


def shuffled_lattice(nc, L, bbks_table, seed=3):
    from tests.helpers import lattice_particles
    p = lattice_particles(nc, L, 9, OM, 0.05, bbks_table)
    return p[np.random.default_rng(seed).permutation(len(p))].copy()


def test_sort_keeps_the_callers_order(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    nc, L = 32, 100.0
    p = shuffled_lattice(nc, L, bbks_table)
    p["x"][:5, 0] = [-0.25, 100.5, 99.999, 0.0, 50.0]          # some wrap
    sim = Simulation(nc, 3 * nc, L, OM)
    sim.set_sort_interval(1)
    sim.set_particles(p, 0.05, 0.05)
    sim.move()                                                  # wrap, then sort
    got = sim.get_particles()
    want = p.copy()
    x = want["x"]
    L32 = np.float32(L)
    want["x"] = np.where(x < 0, x + L32, np.where(x >= L32, x - L32, x)).astype(np.float32)
    for name in PARTICLE_DTYPE.names:
        np.testing.assert_array_equal(got[name], want[name], err_msg=name)
    # a second sort of sorted particles changes nothing either
    sim.move()
    again = sim.get_particles()
    for name in PARTICLE_DTYPE.names:
        np.testing.assert_array_equal(again[name], want[name], err_msg=name)
    sim.close()


def test_sorted_run_matches_unsorted(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.schedule import Schedule
    nc, L = 32, 100.0
    p = shuffled_lattice(nc, L, bbks_table, seed=5)
    out = {}
    for every in (0, 1, 3):
        sim = Simulation(nc, 3 * nc, L, OM)
        sim.set_sort_interval(every)
        sim.set_particles(p, 0.05, 0.05)
        snap = sim.run(Schedule.linear(0.05, 1.0, 6))[-1][1]
        sim.move()
        sim.forces()
        out[every] = (snap, sim.get_forces(), sim.get_particles())
        sim.close()
    s0, f0, p0 = out[0]
    for every in (1, 3):
        s, f, q = out[every]
        np.testing.assert_array_equal(s["id"], s0["id"])
        np.testing.assert_array_equal(q["id"], p0["id"])
        d = np.abs(s["x"] - s0["x"])
        d = np.minimum(d, L - d)
        # the deposit's float sums are added in another order: positions
        # agree to float rounding grown over 6 steps
        assert d.max() < 1e-4 * L, d.max()
        np.testing.assert_allclose(s["v"], s0["v"], rtol=0, atol=2e-3 * np.abs(s0["v"]).max())
        np.testing.assert_allclose(f, f0, rtol=0, atol=2e-3 * np.abs(f0).max())


def test_copy_particles_keeps_the_order(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation, _lib
    nc, L = 16, 50.0
    p = shuffled_lattice(nc, L, bbks_table, seed=8)
    a = Simulation(nc, 2 * nc, L, OM)
    b = Simulation(nc, 2 * nc, L, OM)
    a.set_sort_interval(1)
    a.set_particles(p, 0.05, 0.05)
    a.move()
    _lib.check(gpu_lib.cg_sim_copy_particles(b.h, a.h), "cg_sim_copy_particles")
    pa, pb = a.get_particles(), b.get_particles()
    for name in PARTICLE_DTYPE.names:
        np.testing.assert_array_equal(pb[name], pa[name], err_msg=name)
    a.close()
    b.close()
