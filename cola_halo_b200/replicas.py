"""Realizations across GPUs: one process per GPU, seeds sharded, no
collective on the data path.

The reference runs realizations one after another in one job
(main.c:117-121, seed = random_seed + irealization).  They are independent,
so on N GPUs each rank takes every N-th seed and the only communication is
host-side: a max over ranks of the device time and a gather of the small
per-seed results (P(k), snapshots' summary statistics) at the end.
"""
import os


def rank_world():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base_seed, rank):
    """The seed of rank `rank`'s realization: base + rank, as the reference
    numbers its realizations (main.c:117-121, random_seed + irealization)."""
    return int(base_seed) + int(rank)


def whole_job_rate(units_per_rank, steps, ms_max, world):
    """Throughput of the whole job: every rank processed units_per_rank x
    steps units, and the job took the slowest rank's device time ms_max."""
    if ms_max <= 0:
        raise ValueError("device time must be positive")
    return world * float(units_per_rank) * steps / (ms_max / 1e3)


def shard(items, rank, world):
    """Round-robin share of `items` for `rank` of `world` (seed i -> rank i % world)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank %r / world %r" % (rank, world))
    return list(items)[rank::world]


def allmax(value, dist=None):
    """Max of a float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(local, dist=None):
    """Merge per-rank dicts {seed: result} into one dict on every rank."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, dict(local))
    merged = {}
    for p in parts:
        overlap = set(merged) & set(p)
        if overlap:
            raise RuntimeError("seed computed on two ranks: %s" % sorted(overlap))
        merged.update(p)
    return merged


def run_replicas(seeds, fn, dist=None):
    """Run fn(seed) for this rank's share of seeds; gather all results."""
    if dist is not None and dist.is_initialized():
        rank, world = dist.get_rank(), dist.get_world_size()
    else:
        rank, world = 0, 1
    local = {s: fn(s) for s in shard(seeds, rank, world)}
    return gather_results(local, dist)
