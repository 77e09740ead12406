"""The force step's column-binned deposit (clouds binned by mesh column, each
z-transform CTA building its density lines in shared memory, k_dfz) against
the mesh deposit + z r2c it replaces, and against the oracle restatement of
pm.c (PtoMesh pm.c:229-276 with the buffer copy pm.c:437-445, then the force
pm.c:565-596)."""
import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu

OM = 0.273


def _forces(lib, p, nc, N, L, fused, keep=False):
    from cola_halo_b200 import Simulation
    assert lib.cg_set_force_deposit(1 if fused else 0) == 0
    try:
        sim = Simulation(nc, N, L, OM, np_capacity=max(len(p), 1))
        if keep:
            sim.keep_density(True)
        sim.set_particles(p, 0.1, 0.1)
        sim.move()
        dsum = sim.forces(check_density=True)
        f = sim.get_forces()
        d = sim.get_mesh(0)
        sim.close()
    finally:
        lib.cg_set_force_deposit(-1)
    return f, dsum, d


@pytest.mark.parametrize("nc,factor,L", [(16, 1, 80.0), (16, 3, 100.0), (32, 3, 200.0),
                                         (32, 2, 150.0), (48, 3, 150.0)])
def test_binned_forces_match_mesh_deposit_and_oracle(gpu_lib, bbks_table, nc, factor, L):
    """2LPT particles at a = 0.1; (16, 1) is the mesh of one z tile per plane
    (TY = N), where the wrapped column lies inside the tile."""
    N = nc * factor
    p = lattice_particles(nc, L, 300 + nc, OM, 0.1, bbks_table)
    fb, sb, db = _forces(gpu_lib, p, nc, N, L, True)
    fm, sm, dm = _forces(gpu_lib, p, nc, N, L, False)
    scale = np.abs(fm).max()
    # only the order of the deposit's float additions differs
    assert np.abs(fb - fm).max() < 1e-5 * scale
    assert abs(sb - sm) < 1e-6 * nc ** 3
    x = R.wrap(p["x"], L)
    fo, dens = R.pm_calculate_forces(x, N, L, factor)
    assert np.abs(fb - fo).max() < 2e-5 * scale
    assert np.sqrt(np.mean((fb - fo) ** 2)) < 2e-6 * scale
    s, tol, ok = R.check_total_density(dens.astype(np.float64), factor, nc ** 3)
    assert ok and abs(sb - s) < 1e-6 * nc ** 3
    # the density mesh after a binned step is deposited again on request
    assert np.abs(db - dens).max() < 2e-5 * max(1.0, np.abs(dens).max())


def test_single_particles_bit_identical(gpu_lib):
    """One particle adds once to every cell it reaches in both paths, so the
    spectra and forces agree bit for bit: interior, the last x cell (buffer
    copy), periodic y and z faces, the z tiles' edges (y = 15, 16 cells), and
    x = L or y = L exactly."""
    from cola_halo_b200 import PARTICLE_DTYPE
    nc, factor, L = 16, 3, 48.0
    N = nc * factor
    for xyz in ([10.3, 20.7, 5.5], [47.6, 0.2, 47.9], [0.0, 47.99, 13.0],
                [15.5, 15.9, 31.7], [16.0, 31.999, 47.0], [48.0, 3.3, 7.1], [5.0, 48.0, 0.0],
                [47.99, 47.99, 47.99], [0.001, 15.99, 0.001]):
        p = np.zeros(1, dtype=PARTICLE_DTYPE)
        p["x"] = xyz
        fb, sb, _ = _forces(gpu_lib, p, nc, N, L, True)
        fm, sm, _ = _forces(gpu_lib, p, nc, N, L, False)
        np.testing.assert_array_equal(fb, fm)
        assert sb == sm
        # the mesh holds -1 everywhere plus the particle's mass factor^3
        assert abs(sb - (factor ** 3 - float(N) ** 3)) < 1e-3


def test_dense_clump_and_empty(gpu_lib):
    """Half the particles in one cell's neighbourhood (thousands of clouds in
    a few columns: shared-memory atomics on the same cells), the rest
    uniform, with some in the last x cell; and a force step with no
    particles at all (every line -1)."""
    from cola_halo_b200 import PARTICLE_DTYPE
    nc, factor, L = 16, 3, 100.0
    N = nc * factor
    rng = np.random.default_rng(11)
    n = nc ** 3
    p = np.zeros(n, dtype=PARTICLE_DTYPE)
    xyz = rng.uniform(0.0, L, (n, 3))
    xyz[: n // 2] = np.array([37.3, 99.9, 0.05]) + rng.normal(0.0, 0.4, (n // 2, 3))
    xyz[n // 2: n // 2 + 64, 0] = L - rng.uniform(0.0, L / N, 64)
    p["x"] = np.mod(xyz, L).astype(np.float32)
    fb, sb, _ = _forces(gpu_lib, p, nc, N, L, True)
    fm, sm, _ = _forces(gpu_lib, p, nc, N, L, False)
    scale = np.abs(fm).max()
    assert np.abs(fb - fm).max() < 1e-5 * scale
    fo, _ = R.pm_calculate_forces(R.wrap(p["x"], L), N, L, factor)
    assert np.abs(fb - fo).max() < 2e-5 * scale
    # the clump's cells hold ~10^4: the sums of the float meshes differ by
    # their rounding
    assert abs(sb - sm) < 1e-6 * n * factor ** 3
    # no particles: the density is -1 everywhere, the sum -N^3, no force
    from cola_halo_b200 import Simulation
    sim = Simulation(nc, N, L, OM, np_capacity=8)
    sim.set_particles(np.zeros(0, dtype=PARTICLE_DTYPE), 0.1, 0.1)
    sim.move()
    s = sim.forces(check_density=True)
    assert s == -float(N) ** 3
    assert sim.get_forces().shape[0] == 0
    sim.close()


def test_kept_density_takes_the_mesh_path(gpu_lib, bbks_table):
    """A handle that keeps its density deposits into the mesh, which then is
    the density the force step transformed; the binned default gives the
    same forces to rounding."""
    nc, factor, L = 16, 3, 100.0
    N = nc * factor
    p = lattice_particles(nc, L, 41, OM, 0.1, bbks_table)
    fk, sk, dk = _forces(gpu_lib, p, nc, N, L, True, keep=True)
    fb, sb, db = _forces(gpu_lib, p, nc, N, L, True)
    x = R.wrap(p["x"], L)
    _, dens = R.pm_calculate_forces(x, N, L, factor)
    assert np.abs(dk - dens).max() < 2e-5 * max(1.0, np.abs(dens).max())
    assert np.abs(fk - fb).max() < 1e-5 * np.abs(fk).max()


def test_bad_mode_rejected(gpu_lib):
    assert gpu_lib.cg_set_force_deposit(2) != 0
    assert gpu_lib.cg_set_force_deposit(-1) == 0
