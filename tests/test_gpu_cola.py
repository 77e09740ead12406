"""Kick / drift / wrap / snapshot kernels vs the float32 restatement of
cola.c and move.c: bit-identical given the same inputs and coefficients."""
import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu

OM = 0.273


def _state(n, L, seed):
    rng = np.random.default_rng(seed)
    from cola_halo_b200 import PARTICLE_DTYPE
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    p["x"] = rng.uniform(-0.1 * L, 1.1 * L, (n, 3)).astype(np.float32)
    p["dx1"] = rng.normal(0, 3, (n, 3)).astype(np.float32)
    p["dx2"] = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    p["v"] = rng.normal(0, 2, (n, 3)).astype(np.float32)
    p["id"] = np.arange(1, n + 1)
    return p


def test_wrap_kick_drift_bit_exact(gpu_lib):
    from cola_halo_b200 import Simulation
    nc, L = 16, 100.0
    n = nc ** 3
    p = _state(n, L, 1)
    sim = Simulation(nc, 48, L, OM)
    sim.set_particles(p, 0.3, 0.35)
    sim.move()
    x = R.wrap(p["x"], L)
    np.testing.assert_array_equal(sim.get_particles()["x"], x)
    sim.forces()
    f = sim.get_forces()
    dda, q1, q2 = np.float32(0.71), np.float32(0.4137), np.float32(0.0927)
    sim.kick_coeffs(dda, q1, q2)
    v = R.cola_kick(p["v"], f, p["dx1"], p["dx2"], OM, dda, q1, q2)
    np.testing.assert_array_equal(sim.get_particles()["v"], v)
    dyyy, da1, da2 = np.float32(1.93), np.float32(0.081), np.float32(0.0123)
    sim.drift_coeffs(dyyy, da1, da2)
    xn = R.cola_drift(x, v, p["dx1"], p["dx2"], dyyy, da1, da2)
    np.testing.assert_array_equal(sim.get_particles()["x"], xn)


def test_fused_kick_drift_bit_identical(gpu_lib):
    """cg_sim_kick_drift equals cg_sim_kick followed by cg_sim_drift."""
    from cola_halo_b200 import Simulation
    nc, L = 16, 100.0
    p = _state(nc ** 3, L, 2)
    sim = Simulation(nc, 48, L, OM)
    sim.set_particles(p, 0.3, 0.35)
    sim.move()
    sim.forces()              # float atomics: computed once, used by both paths
    sim.kick(0.4)
    sim.drift(0.45)
    pa, ta = sim.get_particles(), sim.times()
    sim.set_particles(p, 0.3, 0.35)      # same state, the forces stay
    sim.move()
    sim.kick_drift(0.4, 0.45)
    pb, tb = sim.get_particles(), sim.times()
    np.testing.assert_array_equal(pa["x"], pb["x"])
    np.testing.assert_array_equal(pa["v"], pb["v"])
    assert ta == tb


def test_kick_drift_coefficients_match_oracle(gpu_lib):
    """The library's double-precision host coefficients (cola.c:77-134)."""
    from cola_halo_b200 import drift_coeffs, kick_coeffs
    ct = R.ColaTime(OM)
    for a_v, a_x, a1 in [(0.1, 0.1, 0.15), (0.15, 0.2, 0.25), (0.85, 0.9, 0.95), (0.02, 0.02, 0.069)]:
        k = kick_coeffs(OM, a_v, a_x, a1)
        ko = ct.kick_coeffs(a_v, a_x, a1)
        np.testing.assert_allclose(k, ko, rtol=2e-7)
        d = drift_coeffs(OM, a_x, a_v, a1)
        do = ct.drift_coeffs(a_x, a_v, a1)
        np.testing.assert_allclose(d, do, rtol=2e-7, atol=1e-12)


def test_snapshot_bit_exact(gpu_lib, bbks_table):
    from cola_halo_b200 import Simulation
    nc, L = 16, 100.0
    p = lattice_particles(nc, L, 9, OM, 0.1, bbks_table)
    p["v"] = np.random.default_rng(3).normal(0, 1, (nc ** 3, 3)).astype(np.float32)
    sim = Simulation(nc, 48, L, OM)
    sim.set_particles(p, 0.9, 0.95)
    sim.move()
    sim.forces()
    f = sim.get_forces()
    x = sim.get_particles()["x"]
    snap = sim.snapshot(1.0)
    ct = R.ColaTime(OM)
    pos, vel = R.cola_set_snapshot(x, p["v"], f, p["dx1"], p["dx2"], 0.9, 0.95, 1.0, ct)
    np.testing.assert_allclose(snap["x"], pos, rtol=0, atol=2e-5)
    np.testing.assert_allclose(snap["v"], vel, rtol=1e-6, atol=1e-3)
    np.testing.assert_array_equal(snap["id"], p["id"])


def test_dropin_queued_kick_is_exact(gpu_lib):
    """The drop-in queues cola_kick and runs it fused with the cola_drift
    that follows, or before any other call that reads the particles: the
    particles come out bit for bit as the two separate updates give."""
    from cola_halo_b200.sim import drift_coeffs, kick_coeffs
    from cola_halo_b200.types import HostParticles
    nc, L = 16, 100.0
    n = nc ** 3
    om = float(np.float32(OM))
    p = _state(n, L, 3)
    lib = gpu_lib
    lib.cg_dropin_set_abort(0)
    lib.pm_init(48, 3, L, 1.25, None, 0, None, 0)
    hp = HostParticles(nc)
    hp.p[:n] = p
    hp.struct.np_local = n
    hp.struct.a_x, hp.struct.a_v = 0.3, 0.35
    lib.move_particles2(hp.ptr, L, None, 0)
    lib.pm_calculate_forces(hp.ptr)
    assert lib.cg_particles_download(hp.ptr) == 0
    x0, v0 = hp.p["x"][:n].copy(), hp.p["v"][:n].copy()
    f0 = hp.force[:n].copy()
    d1, d2 = p["dx1"], p["dx2"]
    # kick then drift: one fused pass
    lib.cola_kick(hp.ptr, om, 0.4)
    lib.cola_drift(hp.ptr, om, 0.45)
    assert lib.cg_particles_download(hp.ptr) == 0
    v1 = R.cola_kick(v0, f0, d1, d2, om, *kick_coeffs(om, 0.35, 0.3, 0.4))
    x1 = R.cola_drift(x0, v1, d1, d2, *drift_coeffs(om, 0.3, 0.4, 0.45))
    np.testing.assert_array_equal(hp.p["v"][:n], v1)
    np.testing.assert_array_equal(hp.p["x"][:n], x1)
    # a queued kick runs before the next call that reads the particles
    lib.cola_kick(hp.ptr, om, 0.5)
    assert lib.cg_particles_download(hp.ptr) == 0
    v2 = R.cola_kick(v1, f0, d1, d2, om, *kick_coeffs(om, 0.4, 0.45, 0.5))
    np.testing.assert_array_equal(hp.p["v"][:n], v2)
    np.testing.assert_array_equal(hp.p["x"][:n], x1)
    lib.cg_dropin_finalize()
