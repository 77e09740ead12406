"""Isotropic force transfer function T(|n|) in the Green step
(cg_sim_set_force_filters / cg_sim_use_force_filter): the Fourier-space
form of the learned force correction, checked against the oracle's PM force
with the same filter."""
import numpy as np
import pytest

from oracle import restate as R
from tests.helpers import lattice_particles

pytestmark = pytest.mark.gpu
OM = 0.273


def _sim(nc, N, L, p):
    from cola_halo_b200 import Simulation
    sim = Simulation(nc, N, L, OM)
    sim.set_particles(p, 0.1, 0.1)
    sim.move()
    return sim


@pytest.mark.parametrize("nc,factor,L,nk", [(16, 3, 100.0, 9), (32, 2, 64.0, 24)])
def test_filtered_forces_match_oracle(gpu_lib, bbks_table, nc, factor, L, nk):
    N = nc * factor
    p = lattice_particles(nc, L, 40 + nc, OM, 0.1, bbks_table)
    knots = (1.0 + 0.4 * np.sin(np.linspace(0.0, 5.0, nk))).astype(np.float32)
    sim = _sim(nc, N, L, p)
    sim.set_force_filters(knots)
    sim.forces()
    f = sim.get_forces()
    x = R.wrap(p["x"], L)
    _, _, meshes = R.pm_force_meshes(x, N, L, factor, knots)
    for a in range(3):
        m = sim.get_mesh(1 + a)
        assert np.abs(m - meshes[a]).max() < 2e-5 * np.abs(meshes[a]).max()
    fo, _ = R.pm_calculate_forces(x, N, L, factor, knots)
    scale = np.abs(fo).max()
    assert np.abs(f - fo).max() < 2e-5 * scale
    # the filter changed the force (the test is not vacuous)
    f0, _ = R.pm_calculate_forces(x, N, L, factor)
    assert np.abs(f0 - fo).max() > 1e-2 * scale
    sim.close()


def test_identity_scaling_and_selection(gpu_lib, bbks_table):
    """T = 1 is the reference's force bit for bit; T = 2 doubles it exactly
    (power-of-two scaling commutes with every rounding on the path); set
    selection and removal switch between them without a copy."""
    nc, N, L = 16, 48, 100.0
    p = lattice_particles(nc, L, 77, OM, 0.1, bbks_table)
    sim = _sim(nc, N, L, p)
    sim.forces()
    f0 = sim.get_forces()
    sim.set_force_filters(np.stack([np.ones(6), 2 * np.ones(6),
                                    np.linspace(1.0, 0.0, 6)]).astype(np.float32))
    sim.forces()
    np.testing.assert_array_equal(sim.get_forces(), f0)            # set 0 is current
    sim.use_force_filter(1)
    sim.forces()
    np.testing.assert_array_equal(sim.get_forces(), 2 * f0)
    sim.use_force_filter(2)
    sim.forces()
    f2 = sim.get_forces()
    assert np.abs(f2).max() < np.abs(f0).max()
    sim.use_force_filter(-1)
    sim.forces()
    np.testing.assert_array_equal(sim.get_forces(), f0)
    from cola_halo_b200._lib import ColaGpuError
    with pytest.raises(ColaGpuError):
        sim.use_force_filter(3)
    sim.set_force_filters(None)
    with pytest.raises(ColaGpuError):
        sim.use_force_filter(0)
    sim.forces()
    np.testing.assert_array_equal(sim.get_forces(), f0)
    sim.close()


def test_forces_are_linear_in_the_knots(gpu_lib, bbks_table):
    """F(sum_j T_j e_j) = sum_j T_j F(e_j): the basis the least-squares fit
    of the transfer function is built on."""
    nc, N, L = 16, 32, 80.0
    p = lattice_particles(nc, L, 12, OM, 0.1, bbks_table)
    sim = _sim(nc, N, L, p)
    nk = 7
    sim.set_force_filters(np.eye(nk, dtype=np.float32))
    basis = []
    for j in range(nk):
        sim.use_force_filter(j)
        sim.forces()
        basis.append(sim.get_forces().astype(np.float64))
    t = np.linspace(1.3, 0.6, nk).astype(np.float32)
    sim.set_force_filters(t)
    sim.forces()
    f = sim.get_forces()
    want = np.tensordot(t.astype(np.float64), np.array(basis), axes=1)
    assert np.abs(f - want).max() < 1e-5 * np.abs(want).max()
    sim.close()


@pytest.mark.parametrize("kernel", [(2, 0, 0), (4, 0, 0), (0, 1, 0), (0, 0, 1), (0, 0, 2),
                                    (4, 1, 2)])
def test_force_kernels_match_oracle(gpu_lib, bbks_table, kernel):
    """Finite-difference gradients, the discrete Laplacian and the CIC
    window correction (cg_sim_set_force_kernel) against the oracle's force
    with the same tables."""
    nc, factor, L = 16, 3, 100.0
    N = nc * factor
    p = lattice_particles(nc, L, 31, OM, 0.1, bbks_table)
    sim = _sim(nc, N, L, p)
    sim.set_force_kernel(*kernel)
    sim.forces()
    f = sim.get_forces()
    x = R.wrap(p["x"], L)
    _, _, meshes = R.pm_force_meshes(x, N, L, factor, kernel=kernel)
    for a in range(3):
        m = sim.get_mesh(1 + a)
        assert np.abs(m - meshes[a]).max() < 2e-5 * np.abs(meshes[a]).max()
    fo, _ = R.pm_calculate_forces(x, N, L, factor, kernel=kernel)
    scale = np.abs(fo).max()
    assert np.abs(f - fo).max() < 2e-5 * scale
    f0, _ = R.pm_calculate_forces(x, N, L, factor)
    assert np.abs(f0 - fo).max() > 1e-3 * scale          # the mode changed the force
    # back to the reference's kernel, bit for bit
    sim.set_force_kernel(0, 0, 0)
    sim.forces()
    g = sim.get_forces()
    sim2 = _sim(nc, N, L, p)
    sim2.forces()
    np.testing.assert_array_equal(g, sim2.get_forces())
    sim.close()
    sim2.close()


def test_force_kernel_with_filter_matches_oracle(gpu_lib, bbks_table):
    nc, factor, L = 16, 2, 64.0
    N = nc * factor
    p = lattice_particles(nc, L, 9, OM, 0.1, bbks_table)
    knots = np.linspace(1.2, 0.7, 10).astype(np.float32)
    sim = _sim(nc, N, L, p)
    sim.set_force_kernel(4, 0, 2)
    sim.set_force_filters(knots)
    sim.forces()
    f = sim.get_forces()
    fo, _ = R.pm_calculate_forces(R.wrap(p["x"], L), N, L, factor, knots=knots, kernel=(4, 0, 2))
    assert np.abs(f - fo).max() < 2e-5 * np.abs(fo).max()
    from cola_halo_b200._lib import ColaGpuError
    for bad in ((1, 0, 0), (0, 2, 0), (0, 0, 3), (-2, 0, 0)):
        with pytest.raises(ColaGpuError):
            sim.set_force_kernel(*bad)
    sim.close()


def test_fitted_transfer_function_gains_over_the_plain_coarse_mesh(gpu_lib, bbks_table):
    """The Fourier-space learned correction on a small workload (32^3
    particles, coarse 32^3 vs fine 96^3 mesh, 6 steps): least squares on
    forces, then P(k) calibration with the CIC window divided out, both
    trained on two seeds, cut the held-out P(k) error of the coarse run."""
    from cola_halo_b200 import Simulation
    from cola_halo_b200.learned import (_final_positions, _lpt_particles,
                                        calibrate_force_filter, filtered_force, fit_force_filter,
                                        pk_error, power_spectrum_on)
    from cola_halo_b200.schedule import Schedule
    nc, L = 32, 80.0
    sched = Schedule.linear(0.05, 1.0, 6)
    fine = Simulation(nc, 3 * nc, L, OM)
    coarse = Simulation(nc, nc, L, OM)
    lsq = fit_force_filter(coarse, fine, sched, [1, 2], bbks_table, nk=8)
    assert lsq.shape == (sched.nloop - 1, 8) and np.isfinite(lsq).all()
    deconv = Simulation(nc, nc, L, OM)
    deconv.set_force_kernel(0, 0, 2)
    cal, hist = calibrate_force_filter(deconv, fine, sched, [1, 2], bbks_table, nk=8, iters=4)
    assert len(hist) == 4 and min(hist) <= hist[0]
    kmax = 0.5 * np.pi * nc / L
    errs = {"coarse": [], "lsq": [], "cal": []}
    for seed in (11, 12):
        p = _lpt_particles(nc, L, seed, OM, sched.a_init, bbks_table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        k, pf, _ = power_spectrum_on(fine, _final_positions(fine, sched, fine.forces), 1.0)
        for name, sim, force in (("coarse", coarse, None), ("lsq", coarse, lsq),
                                 ("cal", deconv, cal)):
            sim.set_particles(p, sched.a_init, sched.a_init)
            f = sim.forces if force is None else filtered_force(sim, force)
            x = _final_positions(sim, sched, f)
            sim.set_force_filters(None)
            _, pc, _ = power_spectrum_on(fine, x, 1.0)
            errs[name].append(pk_error(k, pc, pf, kmax))
    e = {n: float(np.mean(v)) for n, v in errs.items()}
    assert e["lsq"] < 0.6 * e["coarse"], e
    assert e["cal"] < 0.5 * e["coarse"], e
    for s in (fine, coarse, deconv):
        s.close()


def test_force_kernel_from_the_environment(gpu_lib, bbks_table, tmp_path):
    """COLAGPU_FORCE_KERNEL=g,l,d sets the kernel of every realization a
    process creates (the drop-in's included): a child process with it set
    gives the forces that cg_sim_set_force_kernel gives here."""
    import os
    import subprocess
    import sys
    nc, N, L = 16, 32, 64.0
    p = lattice_particles(nc, L, 4, OM, 0.1, bbks_table)
    np.save(tmp_path / "p.npy", p)
    sim = _sim(nc, N, L, p)
    sim.set_force_kernel(4, 0, 2)
    sim.forces()
    want = sim.get_forces()
    sim.close()
    code = ("import numpy as np, sys; sys.path.insert(0, %r)\n"
            "from cola_halo_b200 import Simulation\n"
            "p = np.load(%r)\n"
            "s = Simulation(%d, %d, %r, %r); s.set_particles(p, 0.1, 0.1); s.move(); s.forces()\n"
            "np.save(%r, s.get_forces())\n"
            % (os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
               str(tmp_path / "p.npy"), nc, N, L, OM, str(tmp_path / "f.npy")))
    env = dict(os.environ, COLAGPU_FORCE_KERNEL="4,0,2")
    r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    np.testing.assert_array_equal(np.load(tmp_path / "f.npy"), want)
