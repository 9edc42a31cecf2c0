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
