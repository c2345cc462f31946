"""Process-group plumbing for multi-GPU runs (one process per GPU).

Blind rotations are independent, so a multi-GPU run shards the work with no
collective on the data path: every rank rotates its own batch against its own
replica of the key (weak scaling). The only collectives are the barrier around
the timed region and one max-reduction of each rank's device time, so the job's
time is that of its slowest rank.

Ranks come from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT), as torchrun sets them.
"""
from __future__ import annotations

import datetime
import os


def env_ranks() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment; (0, 1, 0) when absent."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str, timeout_s: float = 120.0):
    """Joins the process group when WORLD_SIZE > 1 and returns torch.distributed, else None.

    A short timeout makes a rank that never arrives end the others' next
    collective with an error instead of a hang."""
    _, world, _ = env_ranks()
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def weak_seed(base: int, rank: int) -> int:
    """Seed of a rank's own inputs: every rank draws a different batch of the same shape."""
    return base + 1000 * rank


def max_over_ranks(value: float, dist, device) -> float:
    """The largest `value` over all ranks (identity without a process group)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank: int, world: int, seconds: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / seconds
