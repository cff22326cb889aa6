"""CWBVH scenes built on the GPU (rq_build_scene_gpu): a valid CWBVH that the
trace kernels and the oracle traverse identically, every triangle stored
with the host Woop transform's rows (once, or within the split budget when
triangles are pre-split), and the same answers as the host SAH build of the
same mesh (occlusion identical, closest triangles identical up to ties,
disagreements explained in FP64)."""
import numpy as np
import pytest

from adjudicate import _explained, prim_ids

pytestmark = pytest.mark.gpu


def _device_mesh(V, I):
    import torch
    return torch.from_numpy(np.ascontiguousarray(V, np.float32)).cuda(), \
        torch.from_numpy(np.ascontiguousarray(I, np.int32)).cuda()


@pytest.fixture(scope="module", params=[(0, 0, 0), (0, 2, 0), (1, 0, 0), (1, 2, 0), (0, 0, 100), (1, 2, 30)],
                ids=["lbvh", "lbvh-treelets", "ploc", "ploc-treelets", "lbvh-split100", "ploc-treelets-split30"])
def built(rq, request):
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(3, 150_000)
    v, i = _device_mesh(V, I)
    method, passes, budget = request.param
    sc = rq.Scene.build_gpu(v, i, optimize_passes=passes, method=method, split_budget=budget)
    nodes, woop, prim = sc.download()
    return V, I, v, i, sc, nodes, woop, prim, budget


def test_layout_and_woop_rows(rq, built):
    V, I, v, i, sc, nodes, woop, prim, budget = built
    n = I.shape[0]
    ids = prim.reshape(-1, 3)
    refs = ids.shape[0]
    assert woop.shape == (3 * refs, 4) and prim.shape == (3 * refs,)
    assert (ids[:, 1:] == -1).all()
    if budget == 0:
        assert np.array_equal(np.sort(ids[:, 0]), np.arange(n))  # every triangle once
    else:
        # every triangle at least once, the extra references within the budget
        assert np.array_equal(np.unique(ids[:, 0]), np.arange(n))
        assert n < refs <= n + n * budget // 100 + 64
    rows = woop.reshape(-1, 3, 4)
    for slot in np.random.default_rng(0).integers(0, refs, 300):
        t = I[ids[slot, 0]]
        want = rq.woopify(V[t[0]], V[t[1]], V[t[2]])
        assert np.array_equal(rows[slot].view(np.uint32), want.view(np.uint32))
    assert 0 < nodes.shape[0] // 5 <= refs


@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_kernels_and_oracle_agree_on_gpu_tree(rq, po, built, query):
    import torch
    from cwbvh_b200 import workloads as W
    V, I, v, i, sc, nodes, woop, prim, _ = built
    hb = rq.HostBVH(V, I, rq.CWBVH)
    ref = W.DeviceScene(rq.CWBVH, hb, rq.Scene.from_host(hb), v, i, W.diag(V), I.shape[0])
    rays = W.ao_rays(ref, 200_000, seed=17)
    ctx = rq.Context()
    hits = torch.empty((rays.shape[0], 4), device="cuda")
    rq.trace_ordered(ctx, sc, rays, hits, query)
    ctx.check()
    r = rays.cpu().numpy()
    got = hits.cpu().numpy()
    want = po.trace(rq.CWBVH, nodes, woop, r, query == rq.ANY)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))  # same buffers, same order
    # against the host SAH build of the same mesh
    hh = torch.empty_like(hits)
    rq.trace_ordered(ctx, ref.scene, rays, hh, query)
    ctx.check()
    g, h = prim_ids(got, prim), prim_ids(hh.cpu().numpy(), hb.prim_index)
    bad = np.nonzero((g >= 0) != (h >= 0))[0] if query == rq.ANY else np.nonzero(g != h)[0]
    unexplained = [k for k in bad if not _explained(po, r[k], V, I, (int(g[k]), int(h[k])))]
    assert not unexplained, (len(bad), unexplained[:5])
    assert (h >= 0).mean() > 0.1


def test_small_and_invalid_meshes(rq, po):
    import torch
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], np.float32)
    cases = [(I, method) for I in (np.array([[0, 1, 2]], np.int32), np.array([[0, 1, 2], [1, 3, 4]], np.int32))
             for method in (rq.GPU_BUILD_LBVH, rq.GPU_BUILD_PLOC)]
    for I, method in cases:
        v, i = _device_mesh(V, I)
        sc = rq.Scene.build_gpu(v, i, method=method, split_budget=400)
        nodes, woop, prim = sc.download()
        rays = np.zeros((64, 8), np.float32)
        rays[:, 0:3] = [0.2, 0.2, -1.0]
        rays[:, 4:7] = [0.0, 0.0, 1.0]
        rays[:, 7] = 10.0
        hits = torch.empty((64, 4), device="cuda")
        ctx = rq.Context()
        rq.trace_ordered(ctx, sc, torch.from_numpy(rays).cuda(), hits, rq.CLOSEST)
        ctx.check()
        want = po.trace(rq.CWBVH, nodes, woop, rays, False)
        assert np.array_equal(hits.cpu().numpy().view(np.uint32), want.view(np.uint32))
        assert (prim_ids(want, prim) == 0).all()  # the z = 0 triangle
    v, i = _device_mesh(V, np.array([[0, 1, 5]], np.int32))
    for method in (rq.GPU_BUILD_LBVH, rq.GPU_BUILD_PLOC):
        with pytest.raises(rq.RQError, match="INVALID_ARG"):
            rq.Scene.build_gpu(v, i, method=method)
    v, i = _device_mesh(V, np.array([[0, 1, 2]], np.int32))
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.Scene.build_gpu(v, i, method=7)
    for budget in (-1, 401):
        with pytest.raises(rq.RQError, match="INVALID_ARG"):
            rq.Scene.build_gpu(v, i, split_budget=budget)


def test_duplicated_geometry(rq, po):
    """Many identical triangles (every box the same) besides a normal mesh:
    both methods build promptly and trace as the oracle does on their trees;
    every copy is stored."""
    import time
    import torch
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(4, grid=16, n_boxes=10)
    dup = np.repeat(I[:1], 50_000, axis=0)
    I2 = np.concatenate([I, dup]).astype(np.int32)
    v, i = _device_mesh(V, I2)
    rays = np.zeros((4096, 8), np.float32)
    rng = np.random.default_rng(2)
    rays[:, 0:3] = rng.uniform(-0.1, 1.1, (4096, 3))
    d = rng.normal(size=(4096, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = 3.0
    for method in (rq.GPU_BUILD_LBVH, rq.GPU_BUILD_PLOC):
        t0 = time.perf_counter()
        sc = rq.Scene.build_gpu(v, i, method=method)
        torch.cuda.synchronize()
        assert time.perf_counter() - t0 < 20.0
        nodes, woop, prim = sc.download()
        assert np.array_equal(np.sort(prim.reshape(-1, 3)[:, 0]), np.arange(I2.shape[0]))
        hits = torch.empty((4096, 4), device="cuda")
        ctx = rq.Context()
        rq.trace_ordered(ctx, sc, torch.from_numpy(rays).cuda(), hits, rq.CLOSEST)
        ctx.check()
        want = po.trace(rq.CWBVH, nodes, woop, rays, False)
        assert np.array_equal(hits.cpu().numpy().view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("method,budget", [(0, 0), (1, 0), (1, 30)], ids=["lbvh", "ploc", "ploc-split30"])
def test_warp_and_thread_treelets_give_the_same_tree(rq, method, budget):
    """The treelet passes with a warp per treelet (the default) and with one
    thread per treelet give byte-identical scenes."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(4, 200_000)
    v, i = _device_mesh(V, I)
    a = rq.Scene.build_gpu(v, i, optimize_passes=3, method=method, split_budget=budget).download()
    b = rq.Scene.build_gpu(v, i, optimize_passes=3, method=method | rq.GPU_BUILD_THREAD_TREELETS,
                           split_budget=budget).download()
    none = rq.Scene.build_gpu(v, i, optimize_passes=0, method=method, split_budget=budget).download()
    for x, y in zip(a, b):
        assert x.shape == y.shape and np.array_equal(x.view(np.uint32), y.view(np.uint32))
    assert not np.array_equal(a[0].view(np.uint32)[:4096], none[0].view(np.uint32)[:4096])  # the passes did work
