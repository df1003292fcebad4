"""Multi-GPU plumbing: one process per GPU, each extending its own shard of
the workload (weak scaling), and the split of one batch into cell-balanced
contiguous task ranges, one per GPU.  The data path has no collective; the
process group carries only the start/stop barriers and the max-over-ranks of
the measured times."""
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


def task_cells_estimate(tasks):
    """Per-task DP-cell estimate of extension tasks: the banded area
    qlen * min(tlen, 2w + 1) (the rows times the widest band; z-drop and band
    narrowing only shrink it).  Used to balance work, never as a count."""
    import numpy as np
    q = np.maximum(tasks["qlen"].astype(np.int64), 0)
    t = np.maximum(tasks["tlen"].astype(np.int64), 0)
    band = 2 * np.maximum(tasks["w"].astype(np.int64), 0) + 1
    return q * np.minimum(t, band)


def partition_by_cells(tasks, n_parts: int):
    """Bounds b[0..n_parts] (b[0] = 0, b[-1] = len(tasks)) cutting the batch
    into contiguous task ranges of near-equal estimated cells, one per GPU:
    range k is tasks[b[k]:b[k+1]].  Every range holds its share of the cells
    to within one task's estimate."""
    import numpy as np
    n = len(tasks)
    if n_parts < 1:
        raise ValueError("n_parts must be at least 1")
    cum = np.cumsum(task_cells_estimate(tasks)) if n else np.zeros(0, np.int64)
    total = int(cum[-1]) if n else 0
    bounds = [0]
    for k in range(1, n_parts):
        # first task whose cumulative cells reach k/n of the total ends range k-1
        cut = int(np.searchsorted(cum, total * k / n_parts, side="left")) + 1 if total else (n * k) // n_parts
        bounds.append(min(max(cut, bounds[-1]), n))
    bounds.append(n)
    return bounds
