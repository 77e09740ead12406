"""The force step's interpolation from the z c2r's shared tiles (k_zi_interp:
clouds binned by mesh column, each CTA of the z transform interpolating its
plane from the force lines it has just transformed) against the CIC gather
of force_at_particle_locations (pm.c:359-412, with the buffer copies'
forces of pm.c:505-532) on the device's own force meshes, and against the
oracle's whole force."""
import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu

OM = 0.273


def _with_edges(p, L, N, rng):
    """2LPT particles plus clouds on every edge the tiles and bins have: the
    last x cell (buffer copy, plane 0 through i1), the last y cell (the tile
    that wraps to line 0), the last z cell, x = L exactly (no primary cloud),
    and positions 0."""
    from cola_halo_b200 import PARTICLE_DTYPE
    h = L / N
    extra = np.array([[L - 0.3 * h, 0.4 * L, 0.5 * L], [0.3 * L, L - 0.2 * h, 0.7 * L],
                      [0.6 * L, 0.1 * L, L - 0.1 * h], [L - 0.5 * h, L - 0.5 * h, L - 0.5 * h],
                      [0.0, 0.0, 0.0], [np.float32(L), 0.25 * L, 0.75 * L],
                      [0.5 * h, 13.9 * h, 0.5 * L], [0.2 * L, 14.0 * h, 0.3 * L]])
    extra = np.concatenate([extra, rng.uniform(0, L, (64, 3))])
    extra[8:40, 1] = L - rng.uniform(0, h, 32)            # more in the wrapped tile
    extra[40:72, 0] = L - rng.uniform(0, h, 32)           # more buffer copies
    q = np.zeros(len(p) + len(extra), dtype=PARTICLE_DTYPE)
    q[: len(p)] = p
    q["x"][len(p):] = extra.astype(np.float32)
    q["id"][len(p):] = np.arange(len(extra)) + 10 ** 9
    return q


def _run(lib, p, nc, N, L, fused):
    from cola_halo_b200 import Simulation
    assert lib.cg_set_force_interp(1 if fused else 0) == 0
    try:
        sim = Simulation(nc, N, L, OM, np_capacity=len(p))
        sim.set_particles(p, 0.1, 0.1)
        sim.move()
        sim.forces()
        f = sim.get_forces()
        x = sim.get_particles()["x"]
        meshes = [sim.get_mesh(1 + a) for a in range(3)]
        sim.close()
    finally:
        lib.cg_set_force_interp(-1)
    return f, x, meshes


@pytest.mark.parametrize("nc,factor,L", [(16, 1, 80.0), (16, 3, 100.0), (32, 3, 200.0),
                                         (32, 2, 150.0), (64, 3, 200.0), (128, 2, 300.0)])
def test_fused_interp_bit_exact_given_meshes(gpu_lib, bbks_table, nc, factor, L):
    """The fused forces equal, bit for bit, the restated CIC gather of the
    force meshes that the same step's spectra give (cg_sim_get_mesh 1..3
    transforms them after a fused step), edge clouds included; and they
    match the oracle's force."""
    N = nc * factor
    rng = np.random.default_rng(nc * factor)
    p = _with_edges(lattice_particles(nc, L, 500 + nc, OM, 0.1, bbks_table), L, N, rng)
    f, x, meshes = _run(gpu_lib, p, nc, N, L, True)
    for a in range(3):
        np.testing.assert_array_equal(f[:, a], R.cic_interp(x, meshes[a], N, L))
    fo, _ = R.pm_calculate_forces(R.wrap(p["x"], L), N, L, factor)
    scale = np.abs(fo).max()
    assert np.abs(f - fo).max() < 2e-5 * scale


def test_unwrapped_positions(gpu_lib):
    """Positions the force step gets without a wrap: x = L exactly (no
    primary cloud; its buffer copy sits at x = 0, in key row 1), x beyond L,
    x just below 0 (a primary cloud in key row 0).  The fused forces still
    equal the restated gather of the step's own force meshes bit for bit."""
    from cola_halo_b200 import PARTICLE_DTYPE, Simulation
    nc, factor, L = 16, 3, 48.0
    N = nc * factor
    h = L / N
    rng = np.random.default_rng(9)
    xyz = rng.uniform(0.0, L, (300, 3))
    xyz[:40, 0] = L
    xyz[40:80, 0] = L + rng.uniform(0.0, 0.9 * h, 40)
    xyz[80:120, 0] = -rng.uniform(0.0, 0.9 * h, 40)
    xyz[120:160, 0] = L - rng.uniform(0.0, h, 40)
    p = np.zeros(len(xyz), dtype=PARTICLE_DTYPE)
    p["x"] = xyz.astype(np.float32)
    assert gpu_lib.cg_set_force_interp(1) == 0
    try:
        sim = Simulation(nc, N, L, OM, np_capacity=len(p))
        sim.set_particles(p, 0.1, 0.1)
        sim.forces()                       # no move: the positions as given
        f = sim.get_forces()
        for a in range(3):
            np.testing.assert_array_equal(f[:, a], R.cic_interp(p["x"], sim.get_mesh(1 + a), N, L))
        sim.close()
    finally:
        gpu_lib.cg_set_force_interp(-1)


def test_fused_and_mesh_interp_agree(gpu_lib, bbks_table):
    """Both interpolations of one set of particles: the same forces up to
    the deposit's float-addition order (the two runs deposit separately)."""
    nc, factor, L = 32, 3, 200.0
    N = nc * factor
    rng = np.random.default_rng(3)
    p = _with_edges(lattice_particles(nc, L, 77, OM, 0.1, bbks_table), L, N, rng)
    f1, x1, _ = _run(gpu_lib, p, nc, N, L, True)
    f0, x0, _ = _run(gpu_lib, p, nc, N, L, False)
    np.testing.assert_array_equal(x0, x1)
    assert np.abs(f1 - f0).max() < 1e-5 * np.abs(f0).max()


def test_bad_mode_rejected(gpu_lib):
    assert gpu_lib.cg_set_force_interp(3) != 0
    assert gpu_lib.cg_set_force_interp(-1) == 0
