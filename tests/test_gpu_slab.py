"""The slab decomposition on the GPU: the library's cg_sim_slab_* stages for
2 and 3 ranks, held by one process on one GPU (LocalComm: the exchanges are
copies between the ranks' handles, and no rank's kernels wait on another's),
against one handle running the whole force (pm_calculate_forces on one
GPU) and against the oracle.  The rank kernels run one after another; the
collectives of a multi-GPU run are torch.distributed's (TorchComm), whose
exchange logic tests/test_slab_cpu.py checks over gloo."""
import numpy as np
import pytest
import torch

from oracle import restate as R
from tests.test_slab_cpu import _ids, _particles

pytestmark = pytest.mark.gpu

OM = 0.273


def _single(rows, nc, N, L, steps=()):
    from cola_halo_b200 import PARTICLE_DTYPE, Simulation
    p = np.zeros(len(rows), dtype=PARTICLE_DTYPE)
    p["x"] = rows[:, :3]
    p["id"] = _ids(rows)
    sim = Simulation(nc, N, L, OM, np_capacity=len(rows))
    sim.set_sort_interval(0)
    sim.set_particles(p, 0.1, 0.1)
    sim.move()
    dsum = sim.forces(check_density=True)
    for avel1, apos1 in steps:
        sim.kick_drift(avel1, apos1)
        sim.move()
        dsum = sim.forces(check_density=True)
    out = sim.get_particles(), sim.get_forces(), dsum
    sim.close()
    return out


def _slab(rows, nc, N, L, P, steps=()):
    from cola_halo_b200 import Simulation
    from cola_halo_b200.slab import GpuRank, LocalComm, SlabPM
    sims = [Simulation(nc, N, L, OM, np_capacity=len(rows)) for _ in range(P)]
    ranks = [GpuRank(s) for s in sims]
    dev_rows = torch.from_numpy(rows).cuda()
    for r, s in enumerate(sims):
        s.set_particles_ptr(dev_rows.data_ptr() if r == 0 else None, len(rows) if r == 0 else 0,
                            0.1, 0.1)
    pm = SlabPM(ranks, LocalComm(P), "cuda")
    for s in sims:
        s.move()
    pm.exchange_particles()
    dsum = pm.forces()
    for avel1, apos1 in steps:
        for s in sims:
            s.kick_drift(avel1, apos1)
            s.move()
        pm.exchange_particles()
        dsum = pm.forces()
    parts = []
    for r, (s, rk) in enumerate(zip(sims, ranks)):
        lo, hi = pm.x_bounds(r)
        got = s.get_particles()
        assert ((got["x"][:, 0] >= lo) & (got["x"][:, 0] < hi)).all()
        parts.append((got, s.get_forces()))
    for s in sims:
        s.close()
    return parts, dsum


@pytest.mark.parametrize("P", [2, 3])
def test_slab_ranks_match_single_gpu(gpu_lib, bbks_table, P):
    nc, L = 16, 100.0
    N = 3 * nc
    rows = _particles(nc, L, 5, bbks_table)
    ps, fs, ds = _single(rows, nc, N, L)
    parts, dsum = _slab(rows, nc, N, L, P)
    ids = np.concatenate([g["id"] for g, _ in parts])
    f = np.concatenate([fr for _, fr in parts])
    order = np.argsort(ids)
    ref = np.argsort(ps["id"])
    np.testing.assert_array_equal(ids[order], ps["id"][ref])
    scale = np.abs(fs).max()
    # the deposits add in other orders; everything else is the same arithmetic
    assert np.abs(f[order] - fs[ref]).max() < 1e-5 * scale
    assert abs(dsum - ds) < 1e-6 * len(rows)
    fo, _ = R.pm_calculate_forces(R.wrap(rows[:, :3], L), N, L, 3)
    fo_by_id = fo[np.argsort(_ids(rows))]
    assert np.abs(f[order] - fo_by_id).max() < 2e-5 * scale


def test_slab_steps_match_single_gpu(gpu_lib, bbks_table):
    """Three COLA steps (kick + drift, wrap, particles to their slabs, force)
    on 3 ranks against one handle: positions within 1e-5 of the box."""
    nc, L = 16, 100.0
    N = 3 * nc
    rows = _particles(nc, L, 8, bbks_table)
    steps = [(0.15, 0.2), (0.25, 0.3), (0.35, 0.4)]
    ps, fs, _ = _single(rows, nc, N, L, steps)
    parts, _ = _slab(rows, nc, N, L, 3, steps)
    got = np.concatenate([g for g, _ in parts])
    got = got[np.argsort(got["id"])]
    ps = ps[np.argsort(ps["id"])]
    d = np.abs(got["x"].astype(np.float64) - ps["x"])
    d = np.minimum(d, L - d)
    assert d.max() < 1e-5 * L
