"""Seed sharding and result gathering across ranks, world_size 2 on gloo
(CPU): every seed runs on exactly one rank, every rank ends with all
results, and the timing reduction is a max over ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from cola_halo_b200.replicas import allmax, gather_results, run_replicas, shard


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
