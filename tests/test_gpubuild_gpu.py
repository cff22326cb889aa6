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


def _same_tree(a, b) -> int:
    """Walks two CWBVH scenes from the root in slot order and requires the
    same node bytes (all but the child and triangle base offsets, which
    depend on the order the builder's threads allocated the slots in) and
    the same triangles (primitive and Woop rows) in every leaf.  Returns the
    number of nodes compared."""
    na, wa, pa = a
    nb, wb, pb = b
    ua = np.ascontiguousarray(na).view(np.uint32).reshape(-1, 20)
    ub = np.ascontiguousarray(nb).view(np.uint32).reshape(-1, 20)
    wa32 = np.ascontiguousarray(wa).view(np.uint32).reshape(-1, 12)
    wb32 = np.ascontiguousarray(wb).view(np.uint32).reshape(-1, 12)
    pa3, pb3 = pa.reshape(-1, 3), pb.reshape(-1, 3)
    keep = [k for k in range(20) if k not in (4, 5)]  # n1.x child base, n1.y triangle base
    stack, seen = [(0, 0)], 0
    while stack:
        x, y = stack.pop()
        seen += 1
        assert np.array_equal(ua[x, keep], ub[y, keep]), (x, y)
        imask = (int(ua[x, 3]) >> 24) & 0xFF
        meta = int(ua[x, 6]).to_bytes(4, "little") + int(ua[x, 7]).to_bytes(4, "little")
        cb_a, cb_b, tb_a, tb_b = int(ua[x, 4]), int(ub[y, 4]), int(ua[x, 5]), int(ub[y, 5])
        for slot in range(8):
            m = meta[slot]
            if m == 0:
                continue
            if imask & (1 << slot):
                k = bin(imask & ((1 << slot) - 1)).count("1")
                stack.append((cb_a + k, cb_b + k))
            else:
                off, cnt = m & 0x1F, bin(m >> 5).count("1")
                for j in range(cnt):
                    ta, tb = tb_a + off + j, tb_b + off + j
                    assert pa3[ta, 0] == pb3[tb, 0] and np.array_equal(wa32[ta], wb32[tb]), (x, slot, j)
    return seen


@pytest.mark.parametrize("method,budget", [(0, 0), (1, 0), (1, 30)], ids=["lbvh", "ploc", "ploc-split30"])
def test_warp_and_thread_treelets_give_the_same_tree(rq, method, budget):
    """The treelet passes with a warp per treelet (the default) and with one
    thread per treelet give the same tree: node for node and triangle for
    triangle from the root (the builder places nodes in the order its
    threads claim slots, so the offsets differ between builds)."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(4, 200_000)
    v, i = _device_mesh(V, I)
    a = rq.Scene.build_gpu(v, i, optimize_passes=3, method=method, split_budget=budget).download()
    b = rq.Scene.build_gpu(v, i, optimize_passes=3, method=method | rq.GPU_BUILD_THREAD_TREELETS,
                           split_budget=budget).download()
    none = rq.Scene.build_gpu(v, i, optimize_passes=0, method=method, split_budget=budget).download()
    assert a[0].shape[0] // 5 == _same_tree(a, b)  # every node reached and equal
    with pytest.raises((AssertionError, IndexError)):
        _same_tree(a, none)  # the passes changed the tree
