"""Replica execution across the GPUs of one node (one process per GPU, started by
torchrun).

The commitment path shards at job level only: every rank commits its own columns
(seeded at a rank-specific offset of the same counter stream) and proves its own
share of a job list. No data crosses between GPUs, so there is no collective on
the data path; the process group carries only the barrier around a timed region
and the max over ranks of its duration.
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


def env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Joins the process group when there is more than one rank; short timeout so a
    rank that never arrives ends the others with an error instead of a hang."""
    rank, world, local = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local


def barrier() -> None:
    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(x: float, device: torch.device | str | None = None) -> float:
    """Largest value of x over all ranks (the job's time is its slowest replica)."""
    if not dist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard(items, rank: int, world: int) -> list:
    """Round-robin share of a job list for one rank (every job on exactly one rank)."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    return list(items)[rank::world]


def input_offset(rank: int, words_per_rank: int) -> int:
    """Counter offset of a rank's seeded inputs: ranks take consecutive, disjoint
    windows of one SplitMix64 stream (what a single GPU would draw for all of them)."""
    return rank * words_per_rank


def finalize() -> None:
    if dist.is_initialized():
        dist.destroy_process_group()
