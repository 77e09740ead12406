"""The slab decomposition of one realization over ranks
(cola_halo_b200.slab: the reference's comm.c x slabs, pm.c:416-532 buffer
particles, FFTW-MPI transposes, move.c:15-175 particle moves) on CPU: ranks
held by one process (LocalComm) and two gloo processes (TorchComm), each
rank a numpy stand-in for the library's slab stages (tests/slab_cpu_backend).
The assembled forces must match the oracle's undivided PM force
(oracle/restate.py, pm_calculate_forces) and the density sums its
check_total_density sum."""
import os
import socket

import numpy as np
import pytest
import torch

from cola_halo_b200.slab import LocalComm, SlabPM, TorchComm, slab_ranges
from oracle import restate as R
from tests.slab_cpu_backend import CpuRank

OM = 0.273


def _particles(nc, L, seed, table):
    """2LPT particles (a = 0.3) plus clouds on the slab edges of 2 and 3
    ranks and on the periodic face, as n x 14 float32 rows of the reference
    Particle, wrapped into the box."""
    from tests.helpers import lattice_particles
    p = lattice_particles(nc, L, seed, OM, 0.3, table)
    rng = np.random.default_rng(seed)
    N = 3 * nc
    h = L / N
    extra = []
    for P in (2, 3):
        for x0, _ in slab_ranges(N, P):
            for d in (-0.5, -0.01, 0.01, 0.5):
                extra.append([x0 * h + d * h, rng.uniform(0, L), rng.uniform(0, L)])
    extra.append([L - 0.2 * h, 0.5 * L, 0.5 * L])
    x = np.concatenate([R.wrap(p["x"], L), R.wrap(np.array(extra, dtype=np.float32), L)])
    rows = np.zeros((len(x), 14), dtype=np.float32)
    rows[:, :3] = x
    ids = np.arange(1, len(x) + 1, dtype=np.int64)
    rows[:, 12:14] = ids.view(np.float32).reshape(-1, 2)
    return rows


def _ids(rows):
    return np.ascontiguousarray(rows[:, 12:14]).view(np.int64).ravel()


def _check(all_rows, parts, N, L, dsum):
    """parts: (rows, forces) per rank: every particle once, forces as the
    oracle's."""
    ids = np.concatenate([_ids(r) for r, _ in parts])
    assert sorted(ids) == sorted(_ids(all_rows))
    f = np.concatenate([fr.T for _, fr in parts])
    x = np.concatenate([r[:, :3] for r, _ in parts])
    fo, dens = R.pm_calculate_forces(x, N, L, 3)
    scale = np.abs(fo).max()
    assert np.abs(f - fo).max() < 2e-5 * scale
    s, tol, ok = R.check_total_density(dens, 3, len(x))
    assert abs(dsum - s) < 1e-6 * len(x)


@pytest.mark.parametrize("P", [1, 2, 3])
def test_local_ranks_match_oracle(bbks_table, P):
    nc, L = 16, 100.0
    N = 3 * nc
    rows = _particles(nc, L, 5, bbks_table)
    # every particle starts on rank 0; the move sends them to their slabs
    ranks = [CpuRank(N, L, 3, torch.from_numpy(rows if r == 0 else rows[:0])) for r in range(P)]
    pm = SlabPM(ranks, LocalComm(P), "cpu")
    counts = pm.exchange_particles()
    assert sum(counts) == len(rows)
    for r, rk in enumerate(ranks):
        lo, hi = pm.x_bounds(r)
        x = rk.rows[:, 0].numpy()
        assert ((x >= lo) & (x < hi)).all()
    dsum = pm.forces()
    _check(rows, [(rk.rows.numpy(), rk.f.numpy()) for rk in ranks], N, L, dsum)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, table, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nc, L = 16, 100.0
        N = 3 * nc
        rows = _particles(nc, L, 11, table)
        # each rank starts with an interleaved half: most particles move
        mine = torch.from_numpy(rows[rank::world].copy())
        rk = CpuRank(N, L, 3, mine)
        pm = SlabPM([rk], TorchComm(), "cpu")
        pm.exchange_particles()
        dsum = pm.forces()
        q.put((rank, rk.rows.numpy(), rk.f.numpy(), dsum))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_oracle(bbks_table):
    import torch.multiprocessing as mp
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, bbks_table, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted([q.get(timeout=300) for _ in range(world)], key=lambda t: t[0])
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][3] == out[1][3]
    rows = _particles(16, 100.0, 11, bbks_table)
    _check(rows, [(o[1], o[2]) for o in out], 48, 100.0, out[0][3])
