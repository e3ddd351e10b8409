"""Independent replicas on several GPUs (one process per GPU).

The solve has no cross-GPU data exchange: N processes each run the same workload on
their own GPU.  The only collective is the timing reduction -- the whole-job rate is
the units all ranks processed divided by the slowest rank's device time.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def world() -> tuple[int, int]:
    """(rank, world size) of the current process group, (0, 1) without one."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(ms: float, device: torch.device | str = "cpu") -> float:
    """The largest of every rank's value (all ranks must call it, in the same order)."""
    _, n = world()
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if n > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ms_local: float, device: torch.device | str = "cpu") -> tuple[float, float]:
    """(whole-job units per second over all ranks, the slowest rank's milliseconds)."""
    _, n = world()
    ms = max_over_ranks(ms_local, device)
    return units_per_rank * n / (ms / 1e3), ms
