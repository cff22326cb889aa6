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


def shard_range(count: int, world: int, rank: int):
    """(begin, size) of rank `rank`'s contiguous ray range of `count` rays:
    sizes differ by at most one, the larger ranges first (the split of
    rq_shard_range)."""
    if world <= 0 or not 0 <= rank < world or count < 0:
        raise ValueError("bad shard")
    q, r = divmod(count, world)
    return rank * q + min(rank, r), q + (1 if rank < r else 0)


def trace_sharded(trace_range, rays, hits, dist=None):
    """One ray set over the ranks of a process group, each rank holding a
    replica of the scene.  Rank k traces its contiguous range of `rays` with
    `trace_range(rays_slice, hits_slice)` into a local buffer, then the
    ranges are all-gathered so every rank ends with all `hits` (on GPUs an
    NCCL all-gather over NVLink, landing in local memory).  Every rank takes
    the same collective steps whatever its range size: the ranges are padded
    to the largest one for the gather."""
    import torch
    count = rays.shape[0]
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        if count:
            trace_range(rays, hits)
        return hits
    world, rank = dist.get_world_size(), dist.get_rank()
    b, m = shard_range(count, world, rank)
    width = (count + world - 1) // world
    local = torch.zeros((width,) + tuple(hits.shape[1:]), dtype=hits.dtype, device=hits.device)
    if m:
        trace_range(rays[b:b + m], local[:m])
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local)
    for k in range(world):
        bk, mk = shard_range(count, world, k)
        if mk:
            hits[bk:bk + mk].copy_(parts[k][:mk])
    return hits
