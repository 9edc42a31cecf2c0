"""Multi-GPU plumbing for independent reconstructions (one process per GPU).

The path shards by problem: every rank reconstructs its own slices / frames
with no collective on the data path. The only cross-rank steps are the
timing reduction (max over ranks) and the aggregate throughput.
"""

from __future__ import annotations


def rank_seed(base: int, rank: int) -> int:
    """Seed of rank `rank`'s synthetic problems (distinct per rank)."""
    return int(base) + int(rank)


def reduce_max(value: float, device=None) -> float:
    """Max of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, units_per_rank: int, seconds_max: float) -> float:
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max
