"""Replica (multi-GPU) plumbing for independent gridding jobs.

The gridding path has no exchange step: independent jobs (snapshots,
channels) are gridded by independent processes, one per GPU, with no
collective on the data path.  Only the timing needs one: the elapsed time of
a step is the maximum over ranks, and the job throughput is the work of all
ranks divided by it (weak scaling).  These helpers work with any
torch.distributed backend (NCCL on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

import os

import torch


def rank_info():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of the independent job a rank grids."""
    return base_seed + rank


def max_over_ranks(value: float, world_size: int, device="cpu") -> float:
    """Maximum of a per-rank scalar (e.g. elapsed seconds) over all ranks."""
    if world_size <= 1:
        return float(value)
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, world_size: int, device="cpu") -> float:
    if world_size <= 1:
        return float(value)
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def weak_scaling_throughput(points_this_rank: int, steps: int,
                            elapsed_s_this_rank: float, world_size: int,
                            device="cpu") -> float:
    """Visibilities per second of the whole job: every rank's points over
    the slowest rank's time."""
    total = sum_over_ranks(points_this_rank * steps, world_size, device)
    worst = max_over_ranks(elapsed_s_this_rank, world_size, device)
    return total / worst
