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


def _rays(n, seed=1000):
    import numpy as np
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:2] = rng.uniform(0.0, 1.0, (n, 2))
    r[:, 2] = rng.uniform(0.0, 1.2, n)
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 3], r[:, 7] = 1e-4, 0.3
    return r


def _shard_worker(rank, world, port, counts, out):
    import numpy as np
    import torch
    import torch.distributed as dist

    import cwbvh_b200 as rq
    from cwbvh_b200 import replicas
    from cwbvh_b200 import workloads as W
    from oracle import pyoracle as po
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        V, I = W.heightfield_boxes(0)
        hb = rq.HostBVH(V, I, rq.CWBVH)  # every rank holds a replica of the scene
        rays_all = _rays(max(counts))
        traced = []

        def trace_range(r, h):
            traced.append(r.shape[0])
            h.copy_(torch.from_numpy(po.trace(rq.CWBVH, hb.nodes, hb.woop, r.numpy(), True)))

        res = []
        for n in counts:
            rays = torch.from_numpy(rays_all[:n].copy())
            hits = torch.full((n, 4), float("nan"))
            replicas.trace_sharded(trace_range, rays, hits, dist)
            res.append(hits.numpy().copy())
        out.put((rank, traced, res))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_one_ray_set_sharded_over_two_gloo_ranks():
    """Contiguous ray ranges per rank, hits all-gathered: every rank ends with
    the hits of the whole ray set, equal to one process tracing all of it, on
    ragged counts (odd, fewer rays than ranks, none)."""
    import numpy as np

    import cwbvh_b200 as rq
    from cwbvh_b200 import replicas
    from cwbvh_b200 import workloads as W
    from oracle import pyoracle as po
    counts = [4097, 1, 0, 2000]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, counts, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(2)], key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    V, I = W.heightfield_boxes(0)
    hb = rq.HostBVH(V, I, rq.CWBVH)
    rays_all = _rays(max(counts))
    for rank, traced, hits in res:
        # each rank traced only its own contiguous range
        assert traced == [m for m in (replicas.shard_range(n, 2, rank)[1] for n in counts) if m]
        for n, h in zip(counts, hits):
            want = po.trace(rq.CWBVH, hb.nodes, hb.woop, rays_all[:n], True) if n else np.zeros((0, 4), np.float32)
            assert np.array_equal(h.view(np.uint32), want.view(np.uint32))


def test_shard_ranges_cover_the_rays_in_order():
    from cwbvh_b200 import replicas
    for count in (0, 1, 2, 7, 1 << 20, 1_000_003):
        for world in (1, 2, 3, 8):
            rs = [replicas.shard_range(count, world, k) for k in range(world)]
            assert rs[0][0] == 0 and sum(m for _, m in rs) == count
            assert all(rs[k][0] + rs[k][1] == rs[k + 1][0] for k in range(world - 1))
            assert max(m for _, m in rs) - min(m for _, m in rs) <= 1
