"""Converter parity with the reference's ConvertToGPUBVH2 /
ConvertToGPUCompressedWideBVH / WoopifyTriangle (src/GPUBVHConverter.cpp),
pinned by tests/golden/convert_fixtures.npz (made by the reference's own code,
tests/golden/make_golden.py)."""
from pathlib import Path

import numpy as np
import pytest

FIX = Path(__file__).resolve().parent / "golden" / "convert_fixtures.npz"
SCENES = ["hfbox", "flat", "quads", "one_tri", "city"]


@pytest.fixture(scope="module")
def fx():
    return np.load(FIX)


def _tree(fx, name, tag):
    p = f"{name}/{tag}/tree/"
    return {"width": 8 if tag == "cw" else 2, "codes": fx[p + "codes"], "boxes": fx[p + "boxes"],
            "leaf_first": fx[p + "leaf_first"], "leaf_count": fx[p + "leaf_count"],
            "prim_refs": fx[p + "prim_refs"], "root_is_leaf": bool(fx[p + "root_is_leaf"])}


def _woop_close(a, b):
    """Woop rows agree to float rounding of the matrix inverse: the reference
    inverts in float, this library in double."""
    scale = np.maximum(np.abs(b).max(axis=1, keepdims=True), 1e-6)
    return np.abs(a - b) <= 2e-4 * scale


@pytest.mark.parametrize("name", SCENES)
@pytest.mark.parametrize("tag", ["cw", "b2"])
def test_nodes_byte_identical(rq, fx, name, tag):
    V, I = fx[f"{name}/V"], fx[f"{name}/I"]
    hb = rq.HostBVH(V, I, tree=_tree(fx, name, tag))
    ref_nodes = fx[f"{name}/{tag}/ref/nodes"]
    assert hb.nodes.shape == ref_nodes.shape
    assert np.array_equal(hb.nodes.view(np.uint32), ref_nodes.view(np.uint32))
    assert np.array_equal(hb.prim_index, fx[f"{name}/{tag}/ref/prim"])


@pytest.mark.parametrize("name", SCENES)
@pytest.mark.parametrize("tag", ["cw", "b2"])
def test_woop_rows(rq, fx, name, tag):
    V, I = fx[f"{name}/V"], fx[f"{name}/I"]
    hb = rq.HostBVH(V, I, tree=_tree(fx, name, tag))
    ref = fx[f"{name}/{tag}/ref/woop"]
    assert hb.woop.shape == ref.shape
    # Walk the primitive map: a triangle is [prim, -1, -1] (its V0 row
    # first), a BVH2 leaf terminator is a lone -1.
    prim = hb.prim_index
    v0 = np.zeros(prim.size, bool)
    term = np.zeros(prim.size, bool)
    i = 0
    while i < prim.size:
        if prim[i] >= 0:
            v0[i] = True
            i += 3
        else:
            term[i] = True
            i += 1
    bits = hb.woop.view(np.uint32)[:, 0]
    ref_bits = ref.view(np.uint32)[:, 0]
    assert (bits[term] == 0x80000000).all() and (ref_bits[term] == 0x80000000).all()
    # V0.x is never the terminator pattern here (the reference's float
    # inverse can produce -0.0f there, src/TraversalKernelBVH2.cu:132).
    assert not (bits[v0] == 0x80000000).any()
    rows = ~term
    # Compare triangle by triangle (3 rows each).
    a = hb.woop[rows].reshape(-1, 12)
    b = ref[rows].reshape(-1, 12)
    assert _woop_close(a, b).all()


def test_woopify_against_reference(rq, fx):
    tris, ref_rows = fx["woopify/tris"], fx["woopify/ref_rows"]
    for k, t in enumerate(tris):
        mine = rq.woopify(t[0], t[1], t[2])
        if k == 0:
            # Degenerate (collinear): zero rows that no ray can hit; the
            # reference substitutes the identity (a unit triangle at z = 0).
            assert not mine.any()
            assert np.array_equal(ref_rows[k], np.array([[0, 0, 1, -0.0], [1, 0, 0, 0], [0, 1, 0, 0]], np.float32))
            continue
        assert _woop_close(mine.reshape(1, 12), ref_rows[k].reshape(1, 12)).all(), k
        assert mine.view(np.uint32)[0, 0] != 0x80000000  # never a BVH2 leaf terminator


def _decode_cwbvh(nodes):
    """Boxes of every child slot of every CWBVH node: p + q * 2^e."""
    n = nodes.reshape(-1, 5, 4)
    out = []
    for nd in n:
        p = nd[0, :3].astype(np.float64)
        e = nd[0, 3:4].view(np.uint8)[:3].view(np.int8).astype(np.int64)
        q = nd[2:5].reshape(-1).view(np.uint8).reshape(6, 8)  # qlo.x qlo.y qlo.z qhi.x qhi.y qhi.z
        meta = nd[1, 2:4].view(np.uint8)
        scale = np.ldexp(1.0, e)
        lo = p[:, None] + q[0:3] * scale[:, None]
        hi = p[:, None] + q[3:6] * scale[:, None]
        out.append((lo, hi, meta))
    return out


@pytest.mark.parametrize("name", SCENES)
def test_cwbvh_boxes_conservative(rq, fx, name):
    """Every quantised child box contains the child's exact box."""
    V, I = fx[f"{name}/V"], fx[f"{name}/I"]
    tr = _tree(fx, name, "cw")
    hb = rq.HostBVH(V, I, tree=tr)
    # Walk the converted nodes in the converter's order, pairing slots with
    # the tree's boxes through the same greedy slot assignment is not
    # needed: a child's box must be contained in exactly one decoded slot.
    dec = _decode_cwbvh(hb.nodes)
    boxes = tr["boxes"].reshape(-1, 6)
    boxes = boxes[np.isfinite(boxes).all(axis=1) & (tr["codes"].reshape(-1) != -1)]
    all_lo = np.concatenate([d[0].T[d[2] != 0] for d in dec])
    all_hi = np.concatenate([d[1].T[d[2] != 0] for d in dec])
    for b in boxes:
        inside = (all_lo <= b[:3] + 0).all(axis=1) & (all_hi >= b[3:] - 0).all(axis=1)
        assert inside.any()


def test_quantisation_overflow_guard(rq, po):
    """A node whose extent / 255 lies just above a power of two: log2f rounds
    down, and the reference's upper bound rounds up to 256, which its uint8
    store wraps to 0 (src/GPUBVHConverter.cpp:306-316).  The converter here
    takes the next exponent, so the child box stays conservative."""
    ext = np.float32(255.0 * 2.0 ** -7 * (1 + 2.0 ** -22))
    V = np.array([[0, 0, 0], [0.5, 0.1, 0.1], [0.2, 0.3, 0.2],
                  [0.5, 0, 0], [ext, 0.1, 0.1], [0.7, 0.3, 0.2]], np.float32)
    I = np.array([[0, 1, 2], [3, 4, 5]], np.int32)
    codes = np.full((1, 8), -1, np.int32)
    codes[0, 0], codes[0, 1] = -2, -3
    boxes = np.zeros((1, 8, 6), np.float32)
    boxes[0, 0] = [0, 0, 0, 0.5, 0.3, 0.2]
    boxes[0, 1] = [0.5, 0, 0, ext, 0.3, 0.2]
    tree = {"width": 8, "codes": codes, "boxes": boxes, "leaf_first": np.array([0, 1], np.int32),
            "leaf_count": np.array([1, 1], np.int32), "prim_refs": np.array([0, 1], np.int32), "root_is_leaf": False}
    hb = rq.HostBVH(V, I, tree=tree)
    (lo, hi, meta), = _decode_cwbvh(hb.nodes)
    for s in np.nonzero(meta)[0]:
        assert hi[0, s] >= lo[0, s]
    assert hi[0][meta != 0].max() >= ext
    if po.ref_available():
        nodes, _, _ = po.ref_convert(tree, V, I)
        (rlo, rhi, rmeta), = _decode_cwbvh(nodes)
        assert (rhi[0][rmeta != 0] < ext).any()  # the reference's wrapped bound


def test_convert_tree_rejects_bad_trees(rq):
    V = np.zeros((3, 3), np.float32)
    I = np.array([[0, 1, 2]], np.int32)
    codes = np.array([[0, -2, -1, -1, -1, -1, -1, -1]], np.int32)  # the root as its own child
    boxes = np.zeros((1, 8, 6), np.float32)
    bad = {"width": 8, "codes": codes, "boxes": boxes, "leaf_first": np.array([0], np.int32),
           "leaf_count": np.array([1], np.int32), "prim_refs": np.array([0], np.int32), "root_is_leaf": False}
    with pytest.raises(rq.RQError):
        rq.HostBVH(V, I, tree=bad)
    bad["codes"] = np.array([[-1, -2, -1, -1, -1, -1, -1, -1]], np.int32)  # a gap before a child
    with pytest.raises(rq.RQError):
        rq.HostBVH(V, I, tree=bad)
    bad["codes"] = np.array([[-2, -1, -1, -1, -1, -1, -1, -1]], np.int32)
    bad["leaf_count"] = np.array([4], np.int32)  # CWBVH leaves hold at most 3 triangles
    with pytest.raises(rq.RQError):
        rq.HostBVH(V, I, tree=bad)


@pytest.mark.parametrize("presplit", [2, 4, 8])
def test_presplit_keeps_results(rq, po, presplit):
    """Pre-split references change boxes only: every ray gets the same
    occlusion bit and closest triangle, and each leaf lists a triangle once."""
    from cwbvh_b200 import workloads as W
    from adjudicate import prim_ids
    V, I = W.heightfield_boxes(1, grid=24, n_boxes=40)
    rng = np.random.default_rng(4)
    n = 20000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.1, 1.1, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3], rays[:, 7] = 1e-4, 0.3
    base = rq.HostBVH(V, I, rq.CWBVH)
    split = rq.HostBVH(V, I, rq.CWBVH, presplit=presplit)
    tr = split.tree()
    for f, c in zip(tr["leaf_first"], tr["leaf_count"]):
        ids = tr["prim_refs"][f:f + c]
        assert len(set(ids.tolist())) == c
    assert set(tr["prim_refs"].tolist()) == set(range(I.shape[0]))
    for any_hit in (False, True):
        a = prim_ids(po.trace(0, base.nodes, base.woop, rays, any_hit), base.prim_index)
        b = prim_ids(po.trace(0, split.nodes, split.woop, rays, any_hit), split.prim_index)
        assert np.array_equal(a >= 0, b >= 0)
        if not any_hit:
            assert np.array_equal(a, b)


def test_builder_invariants(rq):
    """Leaves hold <= 3 triangles (CWBVH), every triangle is referenced (once
    without spatial splits, at most once per leaf with them), and the depth
    stays within the traversal stacks."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(4, 50_000)
    hb = rq.HostBVH(V, I, rq.CWBVH)
    tr = hb.tree()
    assert tr["leaf_count"].max() <= 3 and tr["leaf_count"].min() >= 1
    assert np.array_equal(np.unique(tr["prim_refs"]), np.arange(I.shape[0]))
    assert tr["prim_refs"].size <= 3 * I.shape[0]
    for f, c in zip(tr["leaf_first"], tr["leaf_count"]):
        assert len(set(tr["prim_refs"][f:f + c].tolist())) == c
    once = rq.HostBVH(V, I, rq.CWBVH, spatial_splits=-1).tree()
    assert np.array_equal(np.sort(once["prim_refs"]), np.arange(I.shape[0]))
    assert 2 * hb.info["depth"] <= 64
    hb2 = rq.HostBVH(V, I, rq.BVH2)
    assert hb2.info["depth"] <= 31


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_build_independent_of_thread_count(rq, kind):
    """The parallel SAH build, 8-wide collapse and conversion give the same
    bytes as the single-threaded ones (subtrees are emitted into precomputed
    ranges)."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(9, 200_000)
    a = rq.HostBVH(V, I, kind, threads=1)
    for th in (3, 8):
        b = rq.HostBVH(V, I, kind, threads=th)
        assert np.array_equal(a.nodes.view(np.uint32), b.nodes.view(np.uint32))
        assert np.array_equal(a.woop.view(np.uint32), b.woop.view(np.uint32))
        assert np.array_equal(a.prim_index, b.prim_index)


def test_treelets_keep_results_and_cut_visits(rq, po):
    """SAH treelet restructuring of the binary tree only rewires inner nodes:
    every AO ray gets the same occlusion bit and the same closest triangle
    (up to ties explained in FP64), every triangle stays referenced once, and
    on the heightfield-and-boxes family far fewer nodes are entered per ray."""
    from cwbvh_b200 import workloads as W
    from adjudicate import _explained, prim_ids
    V, I = W.scene_of_size(3, 150_000)
    rng = np.random.default_rng(6)
    n = 20000
    tri = rng.integers(0, I.shape[0], n)
    a, b = np.sqrt(rng.random(n)), rng.random(n)
    p0, p1, p2 = V[I[tri, 0]], V[I[tri, 1]], V[I[tri, 2]]
    P = p0 * (1 - a)[:, None] + p1 * (a * (1 - b))[:, None] + p2 * (a * b)[:, None]
    Nn = np.cross(p1 - p0, p2 - p0)
    Nn /= np.maximum(np.linalg.norm(Nn, axis=1, keepdims=True), 1e-30)
    pos = np.concatenate([P, np.ones((n, 1))], 1).astype(np.float32)
    nrm = np.concatenate([Nn, np.zeros((n, 1))], 1).astype(np.float32)
    d = W.diag(V)
    rays = po.aorays(pos, nrm, np.zeros(n, np.float32), 1, 7, 1e-4 * d, 0.1 * d, 0.0)
    plain = rq.HostBVH(V, I, rq.CWBVH, treelet_passes=-1, spatial_splits=-1)
    opt = rq.HostBVH(V, I, rq.CWBVH, spatial_splits=-1)  # default passes
    tr = opt.tree()
    assert np.array_equal(np.sort(tr["prim_refs"]), np.arange(I.shape[0]))
    assert tr["leaf_count"].max() <= 3
    for any_hit in (True, False):
        ha, va, _ = po.trace(0, plain.nodes, plain.woop, rays, any_hit, counts=True)
        hb, vb, _ = po.trace(0, opt.nodes, opt.woop, rays, any_hit, counts=True)
        x, y = prim_ids(ha, plain.prim_index), prim_ids(hb, opt.prim_index)
        assert np.array_equal(x >= 0, y >= 0)
        if not any_hit:
            bad = np.nonzero(x != y)[0]
            assert all(_explained(po, rays[k], V, I, (int(x[k]), int(y[k]))) for k in bad), len(bad)
        assert vb.mean() < 0.85 * va.mean(), (vb.mean(), va.mean())


def _ao_rays_numpy(po, V, I, n, seed):
    from cwbvh_b200 import workloads as W
    rng = np.random.default_rng(seed)
    tri = rng.integers(0, I.shape[0], n)
    a, b = np.sqrt(rng.random(n)), rng.random(n)
    p0, p1, p2 = V[I[tri, 0]], V[I[tri, 1]], V[I[tri, 2]]
    P = p0 * (1 - a)[:, None] + p1 * (a * (1 - b))[:, None] + p2 * (a * b)[:, None]
    Nn = np.cross(p1 - p0, p2 - p0)
    Nn /= np.maximum(np.linalg.norm(Nn, axis=1, keepdims=True), 1e-30)
    pos = np.concatenate([P, np.ones((n, 1))], 1).astype(np.float32)
    nrm = np.concatenate([Nn, np.zeros((n, 1))], 1).astype(np.float32)
    d = W.diag(V)
    return po.aorays(pos, nrm, np.zeros(n, np.float32), 1, seed, 1e-4 * d, 0.1 * d, 0.0)


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_spatial_splits_keep_results(rq, po, kind):
    """Spatial splits duplicate references to triangles that straddle a split
    plane, with boxes clipped to each side: every AO ray gets the same
    occlusion bit and the same closest triangle (ties explained in FP64),
    every triangle is still referenced, each duplicate's Woop rows are its
    triangle's, and on the heightfield-and-boxes family fewer nodes are
    entered per ray."""
    from cwbvh_b200 import workloads as W
    from adjudicate import _explained, prim_ids
    V, I = W.scene_of_size(3, 150_000)
    rays = _ao_rays_numpy(po, V, I, 20000, 8)
    plain = rq.HostBVH(V, I, kind, spatial_splits=-1)
    split = rq.HostBVH(V, I, kind, spatial_splits=30)
    if kind == rq.CWBVH:
        tr = split.tree()
        assert tr["leaf_count"].max() <= 3
        n_refs = tr["prim_refs"].size
        assert I.shape[0] < n_refs <= int(1.3 * I.shape[0]) + 1
        assert np.array_equal(np.unique(tr["prim_refs"]), np.arange(I.shape[0]))
        ids = split.prim_index.reshape(-1, 3)[:, 0]
        rows = split.woop.reshape(-1, 3, 4)
        for slot in np.random.default_rng(1).integers(0, ids.size, 200):
            t = I[ids[slot]]
            want = rq.woopify(V[t[0]], V[t[1]], V[t[2]])
            assert np.array_equal(rows[slot].view(np.uint32), want.view(np.uint32))
    for any_hit in (True, False):
        ha, va, _ = po.trace(kind, plain.nodes, plain.woop, rays, any_hit, counts=True)
        hb, vb, _ = po.trace(kind, split.nodes, split.woop, rays, any_hit, counts=True)
        x, y = prim_ids(ha, plain.prim_index), prim_ids(hb, split.prim_index)
        assert np.array_equal(x >= 0, y >= 0)
        if not any_hit:
            bad = np.nonzero(x != y)[0]
            assert all(_explained(po, rays[k], V, I, (int(x[k]), int(y[k]))) for k in bad), len(bad)
        if kind == rq.CWBVH:
            assert vb.mean() < 0.95 * va.mean(), (vb.mean(), va.mean())


def test_spatial_splits_independent_of_thread_count(rq):
    """Slack for duplicates is handed to subtrees in proportion to their
    sizes, so the spatial-split build is the same for any thread count."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(9, 200_000)
    a = rq.HostBVH(V, I, rq.CWBVH, threads=1, spatial_splits=30)
    for th in (3, 8):
        b = rq.HostBVH(V, I, rq.CWBVH, threads=th, spatial_splits=30)
        assert np.array_equal(a.nodes.view(np.uint32), b.nodes.view(np.uint32))
        assert np.array_equal(a.woop.view(np.uint32), b.woop.view(np.uint32))
        assert np.array_equal(a.prim_index, b.prim_index)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.HostBVH(V, I, rq.CWBVH, spatial_splits=1000)


def test_bvh2_treelets_keep_results_within_depth(rq, po):
    """BVH2 builds are restructured too, and the result is kept only while
    the depth stays within the build's limit (31 levels by default, the
    reference BVH2 kernel's stack); answers are unchanged."""
    from cwbvh_b200 import workloads as W
    from adjudicate import _explained, prim_ids
    V, I = W.scene_of_size(3, 150_000)
    rays = _ao_rays_numpy(po, V, I, 20000, 5)
    plain = rq.HostBVH(V, I, rq.BVH2, treelet_passes=-1)
    opt = rq.HostBVH(V, I, rq.BVH2)
    assert opt.info["depth"] <= 31
    for any_hit in (True, False):
        ha, va, _ = po.trace(rq.BVH2, plain.nodes, plain.woop, rays, any_hit, counts=True)
        hb, vb, _ = po.trace(rq.BVH2, opt.nodes, opt.woop, rays, any_hit, counts=True)
        x, y = prim_ids(ha, plain.prim_index), prim_ids(hb, opt.prim_index)
        assert np.array_equal(x >= 0, y >= 0)
        if not any_hit:
            bad = np.nonzero(x != y)[0]
            assert all(_explained(po, rays[k], V, I, (int(x[k]), int(y[k]))) for k in bad), len(bad)
        assert vb.mean() < va.mean()
    shallow = rq.HostBVH(V, I, rq.BVH2, max_depth=20)
    assert shallow.info["depth"] <= 21


def test_large_node_binning_independent_of_thread_count(rq):
    """Nodes of over 1M references are binned on all threads and merged; the
    tree (and so every byte of the scene) is the same as on one thread."""
    from cwbvh_b200 import workloads as W
    V, I = W.scene_of_size(21, 1_100_000)
    a = rq.HostBVH(V, I, rq.CWBVH, threads=1)
    b = rq.HostBVH(V, I, rq.CWBVH, threads=8)
    assert np.array_equal(a.nodes.view(np.uint32), b.nodes.view(np.uint32))
    assert np.array_equal(a.woop.view(np.uint32), b.woop.view(np.uint32))
    assert np.array_equal(a.prim_index, b.prim_index)


def test_spatial_splits_with_degenerate_triangles(rq, po):
    """Zero-area (point and collinear) and duplicated triangles mixed into a
    mesh: the spatial-split build stays valid and answers as the plain build."""
    from cwbvh_b200 import workloads as W
    from adjudicate import prim_ids
    V, I = W.heightfield_boxes(2, grid=24, n_boxes=30)
    rng = np.random.default_rng(3)
    k = 400
    pts = rng.uniform(0, 1, (k, 3)).astype(np.float32)
    base = V.shape[0]
    line = np.concatenate([pts, pts + np.float32(0.05), pts + np.float32(0.1)])  # collinear triples
    V2 = np.concatenate([V, pts, line]).astype(np.float32)
    point_tris = np.stack([base + np.arange(k)] * 3, 1)
    col = base + k + np.arange(k)
    line_tris = np.stack([col, col + k, col + 2 * k], 1)
    dup = I[rng.integers(0, I.shape[0], 200)]
    I2 = np.concatenate([I, point_tris, line_tris, dup]).astype(np.int32)
    rays = _ao_rays_numpy(po, V, I, 10000, 4)
    plain = rq.HostBVH(V2, I2, rq.CWBVH, spatial_splits=-1)
    split = rq.HostBVH(V2, I2, rq.CWBVH, spatial_splits=200)
    tr = split.tree()
    assert np.array_equal(np.unique(tr["prim_refs"]), np.arange(I2.shape[0]))
    for any_hit in (True, False):
        a = prim_ids(po.trace(0, plain.nodes, plain.woop, rays, any_hit), plain.prim_index)
        b = prim_ids(po.trace(0, split.nodes, split.woop, rays, any_hit), split.prim_index)
        assert np.array_equal(a >= 0, b >= 0)


@pytest.mark.parametrize("case", ["soup", "slivers", "tiny", "huge", "coplanar"])
def test_build_options_keep_answers_on_random_meshes(rq, po, case):
    """Spatial splits and treelet restructuring change only the tree: on
    random triangle soups (thin slivers, coordinates near 1e-4 and 1e4, a
    coplanar grid) every ray gets the same occlusion bit and closest
    triangle (up to FP64-explained ties and edges) as the plain SAH build."""
    from adjudicate import _explained, prim_ids
    rng = np.random.default_rng(["soup", "slivers", "tiny", "huge", "coplanar"].index(case) + 11)
    n = 3000
    if case == "coplanar":
        g = 40
        x, y = np.meshgrid(np.arange(g + 1), np.arange(g + 1))
        V = np.stack([x.ravel(), y.ravel(), np.zeros(x.size)], 1).astype(np.float32) / g
        q = (np.arange(g)[:, None] * (g + 1) + np.arange(g)[None, :]).ravel()
        I = np.concatenate([np.stack([q, q + 1, q + g + 2], 1), np.stack([q, q + g + 2, q + g + 1], 1)]).astype(np.int32)
    else:
        c = rng.uniform(0, 1, (n, 3))
        e = rng.normal(size=(n, 2, 3)) * (0.02 if case != "slivers" else np.array([0.002, 0.002, 0.3]))
        V = np.concatenate([c, c + e[:, 0], c + e[:, 1]]).astype(np.float64)
        I = np.stack([np.arange(n), n + np.arange(n), 2 * n + np.arange(n)], 1).astype(np.int32)
        scale = {"tiny": 1e-4, "huge": 1e4}.get(case, 1.0)
        V = (V * scale).astype(np.float32)
    lo, hi = V.min(0), V.max(0)
    m = 8000
    rays = np.zeros((m, 8), np.float32)
    rays[:, 0:3] = rng.uniform(lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo), (m, 3))
    d = rng.normal(size=(m, 3))
    if case == "coplanar":
        rays[:, 2] = 0.5
        d[:, 2] = -np.abs(d[:, 2]) - 0.2
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 0.0
    rays[:, 7] = float(np.linalg.norm(hi - lo)) * 2
    plain = rq.HostBVH(V, I, rq.CWBVH, spatial_splits=-1, treelet_passes=-1)
    opt = rq.HostBVH(V, I, rq.CWBVH)
    for any_hit in (True, False):
        a = prim_ids(po.trace(0, plain.nodes, plain.woop, rays, any_hit), plain.prim_index)
        b = prim_ids(po.trace(0, opt.nodes, opt.woop, rays, any_hit), opt.prim_index)
        bad = np.nonzero((a >= 0) != (b >= 0))[0] if any_hit else np.nonzero(a != b)[0]
        assert all(_explained(po, rays[k], V, I, (int(a[k]), int(b[k]))) for k in bad), (case, any_hit, len(bad))
        assert (b >= 0).mean() > 0.05
