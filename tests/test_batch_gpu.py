"""Batched multi-scene launches: the same answers as per-scene launches and as
the oracle, with and without Morton sorting, eager and CUDA-graph replay."""
import numpy as np
import pytest

from adjudicate import compare, prim_ids

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch_set(rq):
    import torch
    from cwbvh_b200 import workloads as W
    sizes = [(0, 3000, 20000), (1, 40000, 70000), (2, 12000, 0), (3, 800, 1), (4, 25000, 33333)]
    out = []
    for seed, tris, nrays in sizes:
        V, I = W.scene_of_size(seed, tris)
        ds = W.upload(V, I, rq.CWBVH)
        rays = W.ao_rays(ds, max(nrays, 1), seed=seed + 1000)[:nrays].contiguous()
        out.append((V, I, ds, rays))
    torch.cuda.synchronize()
    return out


def _run_batch(rq, ctx, bs, query, **kw):
    import torch
    hits = [torch.full((r.shape[0], 4), float("nan"), device="cuda") for (_, _, _, r) in bs]
    items = [(ds.scene, r, h) for (_, _, ds, r), h in zip(bs, hits)]
    b = rq.Batch(ctx, items, query, **kw)
    s = torch.cuda.Stream()
    b.run(s)
    b.run(s)  # graph replay (when enabled) after the capture run
    s.synchronize()
    ctx.check(s)
    b.close()
    return [h.cpu().numpy() for h in hits]


@pytest.mark.parametrize("sort", [-1, 0, 30000], ids=["unsorted", "sort-all", "sort-large"])
@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_batch_matches_oracle(rq, po, batch_set, sort, graph):
    ctx = rq.Context()
    off = rq.Launch(0, 0, 0, -1.0, 0, 0)  # postponing off: the oracle's order
    for query in (rq.ANY, rq.CLOSEST):
        got = _run_batch(rq, ctx, batch_set, query, launch=off, sort_threshold=sort, use_graph=graph)
        for (V, I, ds, rays), g in zip(batch_set, got):
            r = rays.cpu().numpy()
            want = po.trace(0, ds.host.nodes, ds.host.woop, r, query == rq.ANY)
            assert np.array_equal(g.view(np.uint32), want.view(np.uint32))


def test_batch_production_schedule(rq, po, batch_set):
    """Default launch (postponing on) with sorting: occlusion exact, closest adjudicated."""
    ctx = rq.Context()
    for query in (rq.ANY, rq.CLOSEST):
        got = _run_batch(rq, ctx, batch_set, query, sort_threshold=0, use_graph=True)
        for (V, I, ds, rays), g in zip(batch_set, got):
            r = rays.cpu().numpy()
            want = po.trace(0, ds.host.nodes, ds.host.woop, r, query == rq.ANY)
            res = compare(po, r, g, want, ds.host.prim_index, V, I, query == rq.ANY)
            if query == rq.ANY:
                assert res["disagree"] == 0


def test_batch_equals_plain(rq, batch_set):
    import torch
    ctx = rq.Context()
    got = _run_batch(rq, ctx, batch_set, rq.ANY, sort_threshold=0, use_graph=True)
    for (V, I, ds, rays), g in zip(batch_set, got):
        h = torch.empty((rays.shape[0], 4), device="cuda")
        rq.trace(ctx, ds.scene, rays, h, rq.ANY)
        ctx.check()
        assert np.array_equal(prim_ids(g, ds.host.prim_index) >= 0,
                              prim_ids(h.cpu().numpy(), ds.host.prim_index) >= 0)


def test_batch_stages_and_counts(rq, batch_set):
    import torch
    ctx = rq.Context()
    hits = [torch.empty((r.shape[0], 4), device="cuda") for (_, _, _, r) in batch_set]
    items = [(ds.scene, r, h) for (_, _, ds, r), h in zip(batch_set, hits)]
    b = rq.Batch(ctx, items, rq.ANY, sort_threshold=0, use_graph=True)
    s = torch.cuda.Stream()
    b.run(s)
    s.synchronize()
    full = [h.clone() for h in hits]
    for h in hits:
        h.fill_(0)
    assert rq.lib.rq_batch_run_stage(b._h, 1, s.cuda_stream) == 0
    assert rq.lib.rq_batch_run_stage(b._h, 2, s.cuda_stream) == 0
    s.synchronize()
    ctx.check(s)
    for a, c in zip(full, hits):
        assert torch.equal(a[:, 1].view(torch.int32).ne(-1), c[:, 1].view(torch.int32).ne(-1))
    k = rq.lib.rq_batch_kernel_count(b._h)
    assert k >= 4  # keys + sort passes + gather + trace
    assert rq.lib.rq_batch_total_rays(b._h) == sum(r.shape[0] for (_, _, _, r) in batch_set)


def test_sort_rays_permutation(rq, batch_set):
    import torch
    ctx = rq.Context()
    V, I, ds, rays = batch_set[1]
    lo, hi = ds.host.info["bounds_lo"], ds.host.info["bounds_hi"]
    srt, perm = rq.sort_rays(ctx, rays, lo, hi)
    p = perm.cpu().numpy()
    assert np.array_equal(np.sort(p), np.arange(rays.shape[0]))
    assert torch.equal(srt, rays[perm.long()])


def test_autotune_returns_valid_launch(rq, batch_set, tmp_path):
    import torch
    ctx = rq.Context()
    V, I, ds, rays = batch_set[1]
    hits = torch.empty((rays.shape[0], 4), device="cuda")
    cache = str(tmp_path / "tune.txt")
    l = rq.autotune(ctx, ds.scene, rays, hits, rq.ANY, cache_path=cache)
    assert l.block_size in (64, 128, 256) and l.smem_stack in (4, 8, 16)
    # second stage: refill thresholds from the candidates (Nd -1 stands for 0)
    fetch = {(2, 8), (4, 4), (1, 16), (-1, 1)}
    assert (l.fetch_nd, l.fetch_nw) in fetch
    l2 = rq.autotune(ctx, ds.scene, rays, hits, rq.ANY, cache_path=cache)  # from the cache
    fields = ("block_size", "smem_stack", "postpone_ratio", "fetch_nd", "fetch_nw")
    assert [getattr(l2, f) for f in fields] == [getattr(l, f) for f in fields]
    items = [(d.scene, r, torch.empty((r.shape[0], 4), device="cuda")) for (_, _, d, r) in batch_set]
    bp = rq.autotune_batch(ctx, items, rq.ANY, cache_path=cache, stream=torch.cuda.Stream())
    assert bp.launch.block_size in (64, 128, 256) and bp.use_graph == 1
    assert (bp.launch.fetch_nd, bp.launch.fetch_nw) in fetch
    assert min(abs(bp.launch.postpone_ratio - r) for r in (0.2, 0.3)) < 1e-6
    bp2 = rq.autotune_batch(ctx, items, rq.ANY, cache_path=cache, stream=torch.cuda.Stream())
    assert [getattr(bp2.launch, f) for f in fields] == [getattr(bp.launch, f) for f in fields]
    assert (bp2.sort_threshold, bp2.use_graph) == (bp.sort_threshold, bp.use_graph)
    # the tuned launch traces to the same occlusion as the defaults
    a, b = torch.empty_like(hits), torch.empty_like(hits)
    rq.trace(ctx, ds.scene, rays, a, rq.ANY)
    rq.trace(ctx, ds.scene, rays, b, rq.ANY, launch=l)
    ctx.check()
    assert torch.equal(a[:, 1].view(torch.int32) != -1, b[:, 1].view(torch.int32) != -1)


@pytest.mark.parametrize("graph", [False, True], ids=["eager", "graph"])
def test_ring_batch_matches_oracle(rq, po, graph):
    """An any-hit batch with at least 64 rays per thread of its grid takes the
    kernel that prefetches rays into a ring per warp in shared memory (the
    default large AO batch).  A grid of one 32-thread block per SM reaches it
    with a few hundred thousand rays: in the oracle's order its hits equal the
    oracle's bit for bit, and with the default (full) grid -- the kernel
    without the ring -- they are the same.  Closest-hit batches of the same
    shape (always without the ring) are checked alike."""
    import torch
    from cwbvh_b200 import workloads as W
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    need = 64 * 32 * sms
    sizes = [(10, 5000, need // 3 + 17), (11, 60000, need // 3 + 1), (12, 900, 5), (13, 20000, need // 3 + 4001)]
    bs = []
    for seed, tris, nrays in sizes:
        V, I = W.scene_of_size(seed, tris)
        ds = W.upload(V, I, rq.CWBVH)
        bs.append((V, I, ds, W.ao_rays(ds, nrays, seed=seed + 1000).contiguous()))
    assert sum(r.shape[0] for (_, _, _, r) in bs) >= need
    ctx = rq.Context()
    narrow = rq.Launch(32, 1, 0, -1.0, 0, 0)  # one 32-thread block per SM, oracle order
    full = rq.Launch(0, 0, 0, -1.0, 0, 0)
    for query in (rq.ANY, rq.CLOSEST):
        got = _run_batch(rq, ctx, bs, query, launch=narrow, sort_threshold=-1, use_graph=graph)
        ref = _run_batch(rq, ctx, bs, query, launch=full, sort_threshold=-1, use_graph=graph)
        for (V, I, ds, rays), g, f in zip(bs, got, ref):
            want = po.trace(0, ds.host.nodes, ds.host.woop, rays.cpu().numpy(), query == rq.ANY)
            assert np.array_equal(g.view(np.uint32), want.view(np.uint32))
            assert np.array_equal(f.view(np.uint32), want.view(np.uint32))


def test_ring_single_scene_matches_oracle(rq, po):
    """A single-scene any-hit launch with at least 256 rays per thread of its
    grid takes the ring-prefetching kernel too: bit for bit the oracle's hits
    in its order, and the same as the kernel without the ring (full grid)."""
    import torch
    from cwbvh_b200 import workloads as W
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    n = 256 * 32 * sms + 777
    V, I = W.scene_of_size(21, 30000)
    ds = W.upload(V, I, rq.CWBVH)
    rays = W.ao_rays(ds, n, seed=1021).contiguous()
    ctx = rq.Context()
    got = torch.full((n, 4), float("nan"), device="cuda")
    ref = torch.full((n, 4), float("nan"), device="cuda")
    rq.trace(ctx, ds.scene, rays, got, rq.ANY, launch=rq.Launch(32, 1, 0, -1.0, 0, 0))
    rq.trace(ctx, ds.scene, rays, ref, rq.ANY, launch=rq.Launch(0, 0, 0, -1.0, 0, 0))
    ctx.check()
    want = po.trace(0, ds.host.nodes, ds.host.woop, rays.cpu().numpy(), True)
    assert np.array_equal(got.cpu().numpy().view(np.uint32), want.view(np.uint32))
    assert torch.equal(got.view(torch.int32), ref.view(torch.int32))
