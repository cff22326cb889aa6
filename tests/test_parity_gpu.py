"""CUDA trace kernels against the CPU oracle (the parity gate).

* rq_trace_ordered (no triangle postponing / no speculative leaf postponing)
  must equal the oracle bit for bit: t, Woop address, u, v of every ray.
* rq_trace with the production schedule (warp postponing, dynamic fetch)
  must agree on every occlusion bit / closest primitive id, t within 1e-6
  relative, any disagreement adjudicated in FP64 (tests/adjudicate.py).
"""
import numpy as np
import pytest

from adjudicate import compare

pytestmark = pytest.mark.gpu

N_RAYS = 1 << 20  # config 0's ray count


@pytest.fixture(scope="module")
def small(rq):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    scenes = {k: W.upload(V, I, k) for k in (rq.CWBVH, rq.BVH2)}
    rays = W.ao_rays(scenes[rq.CWBVH], N_RAYS, seed=1000)
    torch.cuda.synchronize()
    return V, I, scenes, rays


def _run(rq, fn, ctx, ds, rays, query, **kw):
    import torch
    hits = torch.full((rays.shape[0], 4), float("nan"), device="cuda")
    fn(ctx, ds.scene, rays, hits, query, **kw)
    ctx.check()
    return hits.cpu().numpy()


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_ordered_bit_exact(rq, po, small, kind, query):
    V, I, scenes, rays = small
    ds = scenes[kind]
    ctx = rq.Context()
    got = _run(rq, rq.trace_ordered, ctx, ds, rays, query)
    r = rays.cpu().numpy()
    want = po.trace(kind, ds.host.nodes, ds.host.woop, r, query == rq.ANY)
    res = compare(po, r, got, want, ds.host.prim_index, V, I, query == rq.ANY, exact=True)
    assert res["hits"] > N_RAYS // 10


@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_slab_extremes_edge_cases_bit_exact(rq, po, small, query):
    """Edge cases of the integer-ordered slab extremes (negative values
    compare in reverse): rays with tmin = 0 and tmin < 0 mixed with ordinary
    ones in every warp, and a scene at 1e15 scale (node exponents and origins
    far beyond the usual range) equal the oracle bit for bit."""
    from cwbvh_b200 import workloads as W
    V, I, scenes, rays = small
    r = rays[:200_000].cpu().numpy().copy()
    r[::3, 3] = 0.0  # tmin = 0 on every third ray
    r[1::7, 3] = -1.0  # and negative on some
    import torch
    ctx = rq.Context()
    cases = [(scenes[rq.CWBVH], V, r)]
    Vb = (V.astype(np.float64) * 1e15).astype(np.float32)
    big = W.upload(Vb, I, rq.CWBVH)
    rb = W.ao_rays(big, 200_000, seed=77).cpu().numpy()
    rb[::4, 3] = 0.0
    cases.append((big, Vb, rb))
    for k, (ds, VV, rr) in enumerate(cases):
        got = _run(rq, rq.trace_ordered, ctx, ds, torch.from_numpy(rr).cuda(), query)
        want = po.trace(rq.CWBVH, ds.host.nodes, ds.host.woop, rr, query == rq.ANY)
        res = compare(po, rr, got, want, ds.host.prim_index, VV, I, query == rq.ANY, exact=True)
        # (at 1e15 the Woop test's float cancellation leaves few or no hits:
        # that scene checks the traversal's node decisions only)
        assert res["hits"] > 0 or k == 1


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_production_schedule_adjudicated(rq, po, small, kind, query):
    V, I, scenes, rays = small
    ds = scenes[kind]
    ctx = rq.Context()
    got = _run(rq, rq.trace, ctx, ds, rays, query)
    r = rays.cpu().numpy()
    want = po.trace(kind, ds.host.nodes, ds.host.woop, r, query == rq.ANY)
    res = compare(po, r, got, want, ds.host.prim_index, V, I, query == rq.ANY)
    if query == rq.ANY:
        assert res["disagree"] == 0  # occlusion does not depend on traversal order


@pytest.mark.parametrize("block", [32, 64, 128, 256, 512])
@pytest.mark.parametrize("smem", [4, 8, 16])
def test_launch_shapes(rq, po, small, block, smem):
    """Every launch shape gives the oracle's occlusion bits exactly."""
    V, I, scenes, rays = small
    ds = scenes[rq.CWBVH]
    ctx = rq.Context()
    l = rq.Launch(block, 0, smem, 0.2, 4, 16)
    got = _run(rq, rq.trace, ctx, ds, rays[:50_000].contiguous(), rq.ANY, launch=l)
    want = po.trace(0, ds.host.nodes, ds.host.woop, rays[:50_000].cpu().numpy(), True)
    assert np.array_equal(got[:, 1].view(np.int32) >= 0, want[:, 1].view(np.int32) >= 0)


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_counts_match_oracle(rq, po, small, kind):
    """Nodes fetched and triangles tested per ray equal the oracle's."""
    import torch
    V, I, scenes, rays = small
    ds = scenes[kind]
    ctx = rq.Context()
    r = rays[:50_000].contiguous()
    for query in (rq.CLOSEST, rq.ANY):
        hits = torch.empty((r.shape[0], 4), device="cuda")
        nv, nt = rq.trace_counted(ctx, ds.scene, r, hits, query)
        ctx.check()
        _, onv, ont = po.trace(kind, ds.host.nodes, ds.host.woop, r.cpu().numpy(), query == rq.ANY, counts=True)
        assert np.array_equal(nv.cpu().numpy(), onv)
        assert np.array_equal(nt.cpu().numpy(), ont)


def _quads(n=1000, r=5000):
    tid = np.arange(n)
    V = np.zeros((3 * n, 3), np.float32)
    V[0::3] = np.stack([np.full(n, -1.1), np.full(n, -1.1), tid], 1)
    V[1::3] = np.stack([np.full(n, 1.1), np.full(n, -1.1), tid], 1)
    V[2::3] = np.stack([np.full(n, 1.1), np.full(n, 1.1), tid], 1)
    I = np.arange(3 * n, dtype=np.int32).reshape(-1, 3)
    rid = np.arange(r, dtype=np.int64)
    k = np.fmod(((rid * 12345678) & 0xFFFFFFFF).astype(np.uint32).view(np.int32).astype(np.int64), n)
    d = np.array([-0.01, 0.5, 1.0])
    d = d / np.linalg.norm(d)
    rays = np.zeros((r, 8), np.float32)
    rays[:, 0], rays[:, 1], rays[:, 2], rays[:, 3] = 0.5, -0.5, k - 0.5, 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 1e20
    expect = np.where(k >= 0, k, np.where(k == -1, 0, -1))
    return V, I, rays, expect


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_known_answer_quad_stack(rq, kind):
    """The reference's validation scene (src/ValidationKernels.cu:6-39): the
    closest hit is the first plane above the origin that the ray crosses."""
    import torch
    from adjudicate import prim_ids
    V, I, rays, expect = _quads()
    hb = rq.HostBVH(V, I, kind)
    sc = rq.Scene.from_host(hb)
    ctx = rq.Context()
    r = torch.from_numpy(rays).cuda()
    for query in (rq.CLOSEST, rq.ANY):
        hits = torch.empty((r.shape[0], 4), device="cuda")
        rq.trace(ctx, sc, r, hits, query)
        ctx.check()
        ids = prim_ids(hits.cpu().numpy(), hb.prim_index)
        if query == rq.CLOSEST:
            assert np.array_equal(ids, expect)
        else:
            assert np.array_equal(ids >= 0, expect >= 0)


def test_edge_cases(rq, po):
    """Empty batch, one ray, axis-parallel and zero-component directions,
    tmin >= tmax, rays starting inside boxes, huge tmax, single-triangle and
    empty scenes."""
    import torch
    from cwbvh_b200 import workloads as W
    ctx = rq.Context()
    V, I = W.heightfield_boxes(3, grid=8, n_boxes=20)
    rng = np.random.default_rng(5)
    n = 4096
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.2, 1.2, (n, 3))
    dirs = rng.normal(size=(n, 3))
    dirs[0:512, 0:2] = 0.0          # straight up / down
    dirs[512:1024, 1:3] = 0.0       # along x
    dirs[1024:1100, 2] = -0.0       # negative zero component
    dirs /= np.maximum(np.linalg.norm(dirs, axis=1, keepdims=True), 1e-30)
    rays[:, 4:7] = dirs
    rays[:, 3] = 0.0
    rays[:, 7] = 10.0
    rays[2000:2100, 3] = 5.0        # tmin > tmax: never hits
    rays[2100:2200, 7] = 3e38       # huge tmax
    rays[2200:2300, 3] = rays[2200:2300, 7] = 1.0  # empty interval
    r = torch.from_numpy(rays).cuda()
    for kind in (rq.CWBVH, rq.BVH2):
        hb = rq.HostBVH(V, I, kind)
        sc = rq.Scene.from_host(hb)
        for query in (rq.CLOSEST, rq.ANY):
            hits = torch.empty((n, 4), device="cuda")
            rq.trace_ordered(ctx, sc, r, hits, query)
            ctx.check()
            want = po.trace(kind, hb.nodes, hb.woop, rays, query == rq.ANY)
            assert np.array_equal(hits.cpu().numpy().view(np.uint32), want.view(np.uint32))
            # empty batch is a no-op
            rq.trace(ctx, sc, r[:0], hits[:0], query)
            ctx.check()
        # one triangle (leaf root) and an empty scene
        for verts, idx in ((V[:3], I[:1] * 0 + np.array([[0, 1, 2]], np.int32)), (V[:3], np.zeros((0, 3), np.int32))):
            hb1 = rq.HostBVH(verts, idx, kind)
            sc1 = rq.Scene.from_host(hb1)
            hits = torch.empty((n, 4), device="cuda")
            rq.trace_ordered(ctx, sc1, r, hits, rq.CLOSEST)
            ctx.check()
            want = po.trace(kind, hb1.nodes, hb1.woop, rays, False)
            assert np.array_equal(hits.cpu().numpy().view(np.uint32), want.view(np.uint32))
