"""Replica bookkeeping for multi-GPU runs.

Nothing on this path is sharded: with N GPUs the benchmark and the solvers
run N independent replicas (one process per GPU, launched by torchrun), each
on its own probe seeds / instances.  The process group carries no data-path
collective; it only synchronises the timed region and reduces the per-rank
device times.  These helpers are backend-agnostic so the same code runs with
NCCL on GPUs and with gloo on the CPU (tests).
"""
from __future__ import annotations

import os


def rank_info():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base: int, rank: int) -> int:
    """Seed of replica `rank`: distinct probe streams per rank, rank 0 keeps
    the single-GPU seed."""
    return int(base) + 1000 * int(rank)


def max_over_ranks(values, dist=None, device="cpu"):
    """Element-wise maximum of a list of floats over all ranks (the timed
    region of a replica run ends when its slowest rank ends)."""
    import torch
    vals = [float(v) for v in values]
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def aggregate_rate(units_per_rank: float, world: int, elapsed_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    if elapsed_max <= 0:
        raise ValueError("elapsed time must be positive")
    return float(units_per_rank) * int(world) / float(elapsed_max)
