"""Multi-GPU plumbing of the benchmark: one process per GPU, each extending
its own shard of the workload (weak scaling).  The data path has no
collective; the process group carries only the start/stop barriers and the
max-over-ranks of the measured times."""
from __future__ import annotations

import os
from typing import Tuple


def dist_env() -> Tuple[int, int, int]:
    """(world_size, rank, local_rank) from the torchrun environment (1, 0, 0 alone)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, dist=None, device=None) -> float:
    """The largest x over all ranks (x itself without a process group): a step
    is as slow as its slowest rank."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, world_size: int, seconds: float) -> float:
    """Units all ranks processed per second, each rank holding units_per_rank."""
    return units_per_rank * world_size / seconds
