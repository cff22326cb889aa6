"""Multi-GPU as replicas: rays are independent and scenes are replicated, so
each rank traces its own copy of the workload (different ray seeds) with no
collective on the data path.  The only communication is the reduction of the
step time to its maximum over ranks, which the throughput is computed from.
"""
from __future__ import annotations

from typing import Optional


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`'s copy of a workload item (distinct per rank)."""
    return base_seed + 100 * rank


def max_over_ranks(value: float, dist=None, device: Optional[str] = None) -> float:
    """Max of a per-rank scalar (e.g. ms per step) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_throughput(units_per_rank: int, world: int, ms_per_step_max: float) -> float:
    """Whole-job units per second: every rank processed `units_per_rank` per
    step and the slowest rank took `ms_per_step_max`."""
    return units_per_rank * world / (ms_per_step_max * 1e-3)
