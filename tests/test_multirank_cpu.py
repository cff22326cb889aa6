"""Replica host logic with two gloo ranks on the CPU: distinct per-rank seeds,
the max-over-ranks step time and the whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from cwbvh_b200 import replicas
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 10.0 + 5.0 * rank           # rank 1 is slower
        m = replicas.max_over_ranks(local_ms, dist)
        thr = replicas.weak_scaling_throughput(1_000_000, world, m)
        seeds = [None] * world
        dist.all_gather_object(seeds, replicas.rank_seed(7, rank))
        out.put((rank, m, thr, seeds))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, thr, seeds in res:
        assert m == 15.0  # the slower rank's time
        assert thr == pytest.approx(2_000_000 / 0.015)
        assert len(set(seeds)) == 2


def test_single_process_is_identity():
    from cwbvh_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.weak_scaling_throughput(10, 1, 1.0) == 10_000
