"""Multi-GPU plumbing for independent reconstructions (one process per GPU).

The path shards by problem: every rank reconstructs its own slices / frames
with no collective on the data path. Problems are split over ranks by a
cost model (``problem_cost``, ``partition``); the only cross-rank steps are
the final gather of the images to one rank (``gather_to_root``), the timing
reductions (max / sum over ranks) and the aggregate throughput.
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


def reduce_sum(value: float, device=None) -> float:
    """Sum of a float over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def world_rank() -> tuple[int, int]:
    """(rank, world size) of the process group, or (0, 1) without one."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def problem_cost(prob, iters: int, toeplitz: bool = True, width: int = 6) -> float:
    """Device work of one reconstruction, in arbitrary units, for balancing.

    ``prob`` holds ``sens`` (X, Y, Z, C) and ``ksp`` (1, R, S, C). With the
    Toeplitz normal an iteration is, per coil, one FFT pair on the twice
    oversampled grid (G = 2X * 2Y [* 2Z] points: ~2 G log2 G); the samples
    are gridded only for the adjoint of the data and the PSF (width^d taps
    each, C + 1 passes). Without it every iteration grids forward and back.
    This is the cost C (G log G + M taps) iters of one pass of the
    reference's slice loop (src/bart.c:202-217), used only to balance shards."""
    import math
    sd = list(prob["sens"].shape) + [1] * 4
    kd = list(prob["ksp"].shape) + [1] * 4
    X, Y, Z, C = (int(v) for v in sd[:4])
    dims = [n for n in (X, Y, Z) if n > 1]
    grid = 1
    for n in dims:
        grid *= 2 * n
    taps = width ** len(dims)
    M = int(kd[1]) * int(kd[2])
    fft = 2.0 * grid * math.log2(max(grid, 2))
    grid_pass = float(M) * taps
    if toeplitz:
        return C * iters * fft + (C + 1) * grid_pass
    return C * iters * (fft + 2.0 * grid_pass) + C * grid_pass


def partition(costs, world: int) -> list[list[int]]:
    """Longest-processing-time split of problems over ranks: the most
    expensive problem first, each to the least-loaded rank (ties to the lower
    index and rank, so every rank computes the same split). Returns each
    rank's problem indices in ascending order; together they are disjoint
    and cover range(len(costs)). LPT's makespan is within 4/3 of optimal."""
    if world < 1:
        raise ValueError("partition: world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shards]


def gather_to_root(local: dict, root: int = 0):
    """Merge every rank's ``{problem index: result}`` on ``root`` (host
    objects through the process group; the final gather of outputs, the only
    exchange of the problem-sharded path). Returns the merged dict on
    ``root`` and None elsewhere; the identity without a process group."""
    import torch.distributed as dist
    rank, world = world_rank()
    if world == 1:
        return dict(local)
    parts = [None] * world if rank == root else None
    dist.gather_object(dict(local), parts, dst=root)
    if rank != root:
        return None
    merged: dict = {}
    for p in parts:
        dup = merged.keys() & p.keys()
        if dup:
            raise RuntimeError(f"gather_to_root: problems {sorted(dup)[:4]} came from two ranks")
        merged.update(p)
    return merged
