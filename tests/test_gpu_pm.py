"""PM force (deposit -> r2c -> Green/gradient -> c2r -> interpolation) on the
GPU vs the oracle restatement of pm.c on the same particles."""
import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu

OM = 0.273


@pytest.mark.parametrize("nc,factor,L", [(16, 3, 100.0), (32, 3, 200.0), (16, 2, 64.0),
                                         (32, 1, 300.0), (48, 3, 150.0)])
def test_forces_match_oracle(gpu_lib, bbks_table, nc, factor, L):
    from cola_halo_b200 import Simulation
    N = nc * factor
    p = lattice_particles(nc, L, 100 + nc, OM, 0.1, bbks_table)
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(p, 0.1, 0.1)
    sim.move()
    dsum = sim.forces(check_density=True)
    f = sim.get_forces()
    x = R.wrap(p["x"], L)
    fo, dens = R.pm_calculate_forces(x, N, L, factor)
    # density mesh
    d = sim.get_mesh(0)
    assert np.abs(d - dens).max() < 2e-5 * max(1.0, np.abs(dens).max())
    s, tol, ok = R.check_total_density(d.astype(np.float64), factor, nc ** 3)
    assert ok and abs(dsum - s) < 1e-6 * nc ** 3
    # force meshes vs the oracle's float64 meshes
    _, _, meshes = R.pm_force_meshes(x, N, L, factor)
    for a in range(3):
        m = sim.get_mesh(1 + a)
        assert np.abs(m - meshes[a]).max() < 2e-5 * np.abs(meshes[a]).max()
    # particle forces
    scale = np.abs(fo).max()
    assert np.abs(f - fo).max() < 2e-5 * scale
    assert np.sqrt(np.mean((f - fo) ** 2)) < 2e-6 * scale


def test_interp_bit_exact_given_mesh(gpu_lib, bbks_table):
    """With the device's own force meshes, the CIC gather (pm.c:370-411 plus
    the buffer copy) is reproduced bit for bit by the restatement."""
    from cola_halo_b200 import Simulation
    nc, factor, L = 16, 3, 100.0
    N = nc * factor
    p = lattice_particles(nc, L, 5, OM, 0.1, bbks_table)
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(p, 0.1, 0.1)
    sim.move()
    sim.forces()
    f = sim.get_forces()
    x = sim.get_particles()["x"]
    for a in range(3):
        fo = R.cic_interp(x, sim.get_mesh(1 + a), N, L)
        np.testing.assert_array_equal(f[:, a], fo)


def test_single_particle_mass(gpu_lib):
    """One particle deposits factor^3 in total (pm.c:216,264-275), also when
    it sits in the last x cell and acts through its buffer copy."""
    from cola_halo_b200 import Simulation
    nc, factor, L = 16, 3, 48.0
    N = nc * factor
    sim = Simulation(nc, N, L, OM, np_capacity=nc ** 3)
    # interior; last x/z cells (buffer copy, periodic z); tile edges (cells
    # 15/16 of the 16^3 deposit tiles); x = L and y = L exactly
    for xyz in ([10.3, 20.7, 5.5], [47.6, 0.2, 47.9], [0.0, 47.99, 13.0],
                [15.5, 15.9, 31.7], [16.0, 31.999, 47.0], [48.0, 3.3, 7.1], [5.0, 48.0, 0.0]):
        p = np.zeros(1, dtype=__import__("cola_halo_b200").PARTICLE_DTYPE)
        p["x"] = xyz
        sim.set_particles(p, 0.1, 0.1)
        sim.forces()
        d = sim.get_mesh(0).astype(np.float64)
        assert abs((d + 1.0).sum() - factor ** 3) < 1e-4
        want = R.cic_deposit(np.array([xyz], dtype=np.float32), N, L, factor)
        assert np.abs(d - want).max() < 1e-6


def test_reset_then_deposit_matches_kept_density(gpu_lib, bbks_table):
    """The force step's z transform leaves -1 in the density mesh and the next
    deposit skips its fill: two force steps in a row (with a kick and drift in
    between) give the same forces as a handle that keeps its density and
    fills before every deposit, and both match the oracle."""
    from cola_halo_b200 import Simulation
    nc, factor, L = 16, 3, 100.0
    N = nc * factor
    p = lattice_particles(nc, L, 77, OM, 0.2, bbks_table)
    runs = []
    for keep in (False, True):
        sim = Simulation(nc, N, L, OM)
        if keep:
            sim.keep_density(True)
        sim.set_particles(p, 0.2, 0.2)
        sim.move()
        sim.forces()
        sim.kick(0.25)
        sim.drift(0.3)
        sim.move()
        sim.forces()
        runs.append((sim.get_forces(), sim.get_particles()["x"]))
        if keep:
            # the kept mesh is the density of the second force step
            d = sim.get_mesh(0)
            _, dens = R.pm_calculate_forces(runs[-1][1], N, L, factor)
            assert np.abs(d - dens).max() < 2e-5 * max(1.0, np.abs(dens).max())
        sim.close()
    (f0, x0), (f1, x1) = runs
    # float atomics: the deposits add in different orders, so the first
    # step's forces, and the positions they drift to, agree to rounding
    assert np.abs(x0 - x1).max() < 1e-6 * L
    scale = np.abs(f1).max()
    assert np.abs(f0 - f1).max() < 1e-5 * scale
    fo, _ = R.pm_calculate_forces(x0, N, L, factor)
    assert np.abs(f0 - fo).max() < 2e-5 * scale


def test_deposit_variants_match_oracle(gpu_lib, bbks_table):
    """Every deposit shape (particles per CTA, shared-memory box, or global
    atomics only) gives the oracle's density to float rounding, and the
    tuner picks one of them."""
    from cola_halo_b200 import Simulation
    nc, factor, L = 32, 3, 200.0
    N = nc * factor
    p = lattice_particles(nc, L, 9, OM, 0.5, bbks_table)
    x = R.wrap(p["x"], L)
    _, dens = R.pm_calculate_forces(x, N, L, factor)
    old = gpu_lib.cg_get_deposit_variant(N)
    try:
        for v in range(gpu_lib.cg_deposit_variants()):
            assert gpu_lib.cg_set_deposit_variant(N, v) == 0
            sim = Simulation(nc, N, L, OM)
            sim.keep_density(True)
            sim.set_particles(p, 0.5, 0.5)
            sim.move()
            sim.forces()
            d = sim.get_mesh(0)
            assert np.abs(d - dens).max() < 2e-5 * max(1.0, np.abs(dens).max()), v
            sim.close()
        sim = Simulation(nc, N, L, OM)
        sim.set_particles(p, 0.5, 0.5)
        sim.move()
        from cola_halo_b200.tune import tune_deposit
        best, ms = tune_deposit(sim)
        assert 0 <= best < len(ms) and gpu_lib.cg_get_deposit_variant(N) == best
        assert min(ms) == ms[best]
        sim.close()
    finally:
        gpu_lib.cg_set_deposit_variant(N, old)
    assert gpu_lib.cg_set_deposit_variant(N, 99) != 0
