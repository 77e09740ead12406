"""The gathers of the strided passes run the same arithmetic, so the force
meshes and forces they give are bit-identical: for the z c2r, cp.async, TMA
into a landing area and TMA into the transform's own 128-byte-swizzled
tile; for the x pass, direct loads and TMA into a 64- or 128-byte-swizzled
tile.  The particles sit near the lattice at factor 3, so no two CIC clouds
share a cell and the float-atomic deposit is itself deterministic."""
import numpy as np
import pytest

from oracle import restate as R

pytestmark = pytest.mark.gpu
OM = 0.273


def _particles(nc, L):
    """Lattice q = (i + 1/2) L / nc moved by less than 0.4 mesh cells (mesh
    cell L / (3 nc)): every CIC cloud stays inside its own 3^3 block."""
    from cola_halo_b200.types import PARTICLE_DTYPE
    q = (np.arange(nc) + 0.5) * L / nc
    x = np.stack(np.meshgrid(q, q, q, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(nc)
    x = x + rng.uniform(-0.4, 0.4, x.shape) * L / (3 * nc)
    p = np.zeros(nc ** 3, dtype=PARTICLE_DTYPE)
    p["x"] = x.astype(np.float32)
    p["id"] = np.arange(1, nc ** 3 + 1)
    return p


def _force_run(lib, mode, nc, L, table, meshes, xmode=-1, fx_variant=None, factor=3):
    from cola_halo_b200 import Simulation
    assert lib.cg_set_z_gather(mode) == 0
    assert lib.cg_set_x_gather(xmode) == 0
    if fx_variant is not None:
        assert lib.cg_set_schedule(factor * nc, 0, fx_variant) == 0
    try:
        sim = Simulation(nc, factor * nc, L, OM)
    finally:
        lib.cg_set_z_gather(-1)
        lib.cg_set_x_gather(-1)
    sim.set_particles(_particles(nc, L), 0.02, 0.02)
    sim.move()
    sim.forces()
    out = [sim.get_forces()]
    if meshes:
        out += [sim.get_mesh(a) for a in (1, 2, 3)]
    sim.close()
    return out


@pytest.mark.parametrize("nc,L", [(16, 100.0), (32, 200.0), (64, 200.0), (128, 300.0)])
def test_z_gathers_bit_identical(gpu_lib, bbks_table, nc, L):
    runs = [_force_run(gpu_lib, m, nc, L, bbks_table, True) for m in (0, 1, 2)]
    for other in runs[1:]:
        for a, b in zip(runs[0], other):
            np.testing.assert_array_equal(a, b)
    if nc <= 32:
        fo, _ = R.pm_calculate_forces(R.wrap(_particles(nc, L)["x"], L), 3 * nc, L, 3)
        assert np.abs(runs[2][0] - fo).max() < 2e-5 * np.abs(fo).max()


@pytest.mark.parametrize("nc,L,fxv", [(16, 100.0, None), (32, 200.0, None), (128, 300.0, 0),
                                      (128, 300.0, 2)])
def test_x_gathers_bit_identical(gpu_lib, bbks_table, nc, L, fxv):
    """fxv: the x-pass schedule variant (0: 8 columns per CTA, 64-byte rows;
    2: 16 columns, 128-byte rows), None below 256 where only one exists."""
    try:
        runs = [_force_run(gpu_lib, 2, nc, L, bbks_table, True, xmode=m, fx_variant=fxv)
                for m in (0, 1)]
    finally:
        if fxv is not None:
            gpu_lib.cg_set_schedule(3 * nc, 0, 0)
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)


def test_gathers_bit_identical_768(gpu_lib, bbks_table):
    """The one-GPU workload's mesh: forces of every particle, the plainest
    gathers against the TMA ones."""
    f = [_force_run(gpu_lib, z, 256, 600.0, bbks_table, False, xmode=x)[0]
         for z, x in ((0, 0), (2, 1))]
    np.testing.assert_array_equal(f[0], f[1])


def test_z_gathers_bit_identical_1024(gpu_lib, bbks_table):
    """The large configuration's 1024^3 mesh, where the swizzled TMA z c2r
    reads its twiddles from a shared-memory pack: forces of every particle
    as with the cp.async gather, which reads them from the table.  64^3
    particles at factor 16: the clouds share no cell."""
    f = [_force_run(gpu_lib, z, 64, 1200.0, bbks_table, False, factor=16)[0] for z in (0, 2)]
    assert np.abs(f[0]).max() > 0
    np.testing.assert_array_equal(f[0], f[1])


def test_bad_gather_mode_rejected(gpu_lib):
    assert gpu_lib.cg_set_z_gather(3) != 0
    assert gpu_lib.cg_set_z_gather(-1) == 0
    assert gpu_lib.cg_set_x_gather(2) != 0
    assert gpu_lib.cg_set_x_gather(-1) == 0
