"""Multi-GPU plumbing of the query path: replicas only.

Queries are independent and every index fits one B200, so N GPUs run N
replicas: each rank (one process per GPU, torch.distributed for plumbing)
holds the whole index and answers its own queries. There is no collective on
the data path; the only cross-rank steps are the barriers around the timed
region, the maximum of the per-rank device times and, for checking, gathering
results.
"""
from __future__ import annotations

import os
from dataclasses import dataclass


@dataclass(frozen=True)
class RankInfo:
    rank: int
    world: int
    local_rank: int


def rank_info() -> RankInfo:
    return RankInfo(int(os.environ.get("RANK", "0")),
                    int(os.environ.get("WORLD_SIZE", "1")),
                    int(os.environ.get("LOCAL_RANK", "0")))


def shard(count: int, rank: int, world: int) -> range:
    """The contiguous share of `count` items that `rank` answers (the shares
    of all ranks partition range(count), sizes differ by at most one)."""
    base, extra = divmod(count, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world: int, max_seconds: float) -> float:
    """Units processed by all ranks per second of the slowest rank."""
    return units_per_rank * world / max_seconds
