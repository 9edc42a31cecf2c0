"""World-size-2 run of the multi-GPU host logic on CPU (gloo)."""

import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from bart_b200.dist import aggregate_rate, rank_seed, reduce_max
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seed = rank_seed(1000, rank)
        local_ms = 10.0 + 5.0 * rank          # rank 1 is the slow one
        ms_max = reduce_max(local_ms)
        rate = aggregate_rate(world, 20, ms_max / 1e3)
        q.put((rank, seed, ms_max, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_max_time_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29511
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, m0, v0), (r1, s1, m1, v1) = res
    assert s0 != s1                      # independent problems per rank
    assert m0 == m1 == 15.0              # max over ranks
    assert v0 == v1 == pytest.approx(2 * 20 / 0.015)


def _costs(n, seed):
    import random
    rnd = random.Random(seed)
    return [rnd.random() ** 3 * 100 for _ in range(n)]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_disjoint_complete_balanced(world):
    from bart_b200.dist import partition
    costs = _costs(97, world)
    shards = partition(costs, world)
    assert len(shards) == world
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(costs)))            # every problem once
    assert all(s == sorted(s) for s in shards)
    loads = [sum(costs[i] for i in s) for s in shards]
    # LPT bound: makespan <= mean load + the largest single cost
    assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
    assert partition(costs, world) == shards          # deterministic: every rank agrees


def test_partition_more_ranks_than_problems():
    from bart_b200.dist import partition
    shards = partition([3.0, 1.0], 4)
    assert shards == [[0], [1], [], []]
    with pytest.raises(ValueError):
        partition([1.0], 0)


def test_problem_cost_grows_with_size_coils_and_iterations():
    import numpy as np
    from bart_b200.dist import problem_cost

    def prob(N, C, spokes, Z=1):
        return {"sens": np.zeros((N, N, Z, C), np.complex64), "ksp": np.zeros((1, 2 * N, spokes, C), np.complex64)}

    base = problem_cost(prob(128, 8, 64), 20)
    assert problem_cost(prob(256, 8, 64), 20) > 4 * base * 0.9
    assert problem_cost(prob(128, 16, 64), 20) > 1.9 * base
    assert problem_cost(prob(128, 8, 64), 40) > 1.5 * base
    assert problem_cost(prob(128, 8, 64), 20, toeplitz=False) > base
    assert problem_cost(prob(32, 4, 16, Z=32), 20) > problem_cost(prob(32, 4, 16), 20)


def _gather_worker(rank, world, port, q):
    import torch.distributed as dist
    from bart_b200.dist import gather_to_root, partition, reduce_sum, world_rank
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = _costs(23, 5)
        assert world_rank() == (rank, world)
        mine = partition(costs, world)[rank]
        total = reduce_sum(len(mine))
        got = gather_to_root({i: ("img", i, rank) for i in mine})
        q.put((rank, mine, got, total))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather_to_root():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, 29513, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, mine0, got0, n0), (_, mine1, got1, n1) = res
    assert n0 == n1 == 23                             # sum over ranks
    assert got1 is None                               # only the root holds the images
    assert sorted(got0) == list(range(23))
    assert not set(mine0) & set(mine1)
    for i, (tag, idx, r) in got0.items():
        assert tag == "img" and idx == i and i in (mine0 if r == 0 else mine1)


def test_gather_to_root_refuses_a_problem_from_two_ranks(monkeypatch):
    """A split that gave one problem to two ranks is an error on the root,
    not a silent overwrite (the gather itself is faked here)."""
    import torch.distributed as dist
    from bart_b200 import dist as bd
    monkeypatch.setattr(bd, "world_rank", lambda: (0, 2))

    def fake_gather(obj, parts, dst=0):
        parts[0], parts[1] = obj, {1: "b", 2: "c"}

    monkeypatch.setattr(dist, "gather_object", fake_gather)
    assert bd.gather_to_root({0: "a"}) == {0: "a", 1: "b", 2: "c"}
    with pytest.raises(RuntimeError):
        bd.gather_to_root({2: "a"})
