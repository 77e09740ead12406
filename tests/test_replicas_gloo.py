"""Seed sharding and result gathering across ranks, world_size 2 on gloo
(CPU): every seed runs on exactly one rank, every rank ends with all
results, and the timing reduction is a max over ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cola_halo_b200.replicas import (allmax, gather_results, replica_seed, run_replicas,
                                     shard, whole_job_rate)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = list(range(100, 111))
        res = run_replicas(seeds, lambda s: {"seed": s, "rank": rank, "pk0": 1.0 / s}, dist)
        t = allmax(1.0 + rank, dist)
        q.put((rank, sorted(res), {s: r["rank"] for s, r in res.items()}, t))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, seeds, owner, t in out:
        assert seeds == list(range(100, 111))
        assert all(owner[s] == (s - 100) % world for s in seeds)
        assert t == 2.0


def test_shard_and_gather_single():
    assert shard(range(5), 1, 2) == [1, 3]
    with pytest.raises(ValueError):
        shard(range(5), 2, 2)
    assert gather_results({1: "a"}) == {1: "a"}


def _bench_worker(rank, world, port, q):
    """The replica path of bench.py on CPU: each rank runs its own seed
    (replica_seed) through the oracle's 2LPT and two PM force steps at 16^3,
    times it, takes the max over ranks (allmax) and forms the whole-job rate
    (whole_job_rate); the per-seed results are gathered on every rank."""
    import time
    import numpy as np
    from cola_halo_b200.bbks import write_bbks_table
    from oracle import restate as R
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        nc, L, om, a = 16, 100.0, 0.273, 0.5
        seed = replica_seed(100, rank)
        table = write_bbks_table("/tmp/bbks_rank%d_%d.dat" % (rank, port))
        t0 = time.perf_counter()
        o = R.lpt_set_displacement(nc, L, seed, om, a, R.PowerTable(table))
        x = R.wrap(o["x"], L)
        for _ in range(2):
            f, _ = R.pm_calculate_forces(x, 3 * nc, L, 3)
            x = R.wrap((x + 0.01 * f).astype(np.float32), L)
        ms = (time.perf_counter() - t0) * 1e3 * (1 + rank)     # rank 1 twice as slow
        ms_max = allmax(ms, dist)
        rate = whole_job_rate(nc ** 3, 2, ms_max, world)
        res = gather_results({seed: float(np.abs(f).max())}, dist)
        q.put((rank, seed, ms, ms_max, rate, res))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_bench_replica_path():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_bench_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=300) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    seeds = [o[1] for o in out]
    assert seeds == [100, 101]
    slowest = max(o[2] for o in out)
    for rank, seed, ms, ms_max, rate, res in out:
        assert ms_max == slowest
        assert abs(rate - world * 16 ** 3 * 2 / (slowest / 1e3)) < 1e-6 * rate
        assert sorted(res) == [100, 101] and all(v > 0 for v in res.values())
