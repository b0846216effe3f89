"""Multi-GPU host logic: the KT step shards by event (one event per rank, no collective in
the step). torch.distributed is only the plumbing for the barrier and the job timing,
which is the maximum over ranks."""
from __future__ import annotations

import os


def rank_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (defaults: one process)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def event_seed(base_seed: int, rank: int) -> int:
    """Each rank advances its own event; events differ only by their seed."""
    return base_seed + rank


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The job's time is the slowest rank's (all_reduce MAX). `dist` is torch.distributed
    when initialised, else the value is returned unchanged."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(cells_per_rank: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job cell-updates/s: every rank's cells times steps over the slowest rank's time."""
    return world * cells_per_rank * steps / (ms_max / 1e3)
