"""Failure paths of the trace kernels, made with scene buffers that the
kernels' own checks turn into errors (no GPU fault is involved): every node
and triangle address is bounds-checked before its load, the stack before a
push, and a ray that keeps walking ends at the step limit.  The affected rays
come back as misses, rq_ctx_check reports the error once, and the context
keeps working.  (The oracle is not run on these scenes: it has no step
limit.)"""
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def cw_node(child_base, tri_base, imask, metas, full_slots, e=(0, 0, 0), p=(0.0, 0.0, 0.0)):
    """One 80 B CWBVH node; the boxes of `full_slots` span the whole node."""
    b = bytearray(80)
    struct.pack_into("<3f", b, 0, *p)
    b[12:15] = bytes(np.array(e, np.int8).view(np.uint8))
    b[15] = imask
    struct.pack_into("<ii", b, 16, child_base, tri_base)
    for slot, m in metas.items():
        b[24 + slot] = m
    for c in full_slots:
        for a in range(3):
            b[32 + c + 8 * a] = 0          # qlo
            b[32 + c + 8 * (3 + a)] = 255  # qhi
    return np.frombuffer(bytes(b), np.float32).reshape(5, 4)


def rays_inside(n, seed=0):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(50, 200, (n, 3))
    d = rng.normal(size=(n, 3))
    r[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 7] = 1e3
    return r


INNER0, INNER1, LEAF1 = 0x38, 0x39, 0x20  # inner child in slot 0 / 1; one triangle at offset 0


def _trace(rq, ctx, scene, rays, query, launch=None):
    import torch
    r = torch.from_numpy(rays).cuda()
    hits = torch.full((rays.shape[0], 4), float("nan"), device="cuda")
    rq.trace(ctx, scene, r, hits, query, launch=launch)
    return hits.cpu().numpy()


def _valid_after(rq, ctx):
    """The context still traces a valid scene without error."""
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0, grid=8, n_boxes=4)
    ds = W.upload(V, I, rq.CWBVH)
    rays = W.ao_rays(ds, 4096, seed=3)
    import torch
    hits = torch.empty((4096, 4), device="cuda")
    rq.trace(ctx, ds.scene, rays, hits, rq.ANY)
    ctx.check()


@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_cycle_ends_at_step_limit(rq, query):
    # node 0's only child is node 0 itself: no stack growth, endless walk
    nodes = cw_node(0, 0, 0x01, {0: INNER0}, [0])
    scene = rq.Scene.from_arrays(rq.CWBVH, nodes, np.zeros((3, 4), np.float32))
    ctx = rq.Context()
    hits = _trace(rq, ctx, scene, rays_inside(64), query, launch=rq.Launch(0, 0, 0, 0.0, 0, 0, 2000))
    with pytest.raises(rq.RQError, match="TIMEOUT"):
        ctx.check()
    assert (hits[:, 1].view(np.int32) == -1).all()
    ctx.check()  # reported once
    _valid_after(rq, ctx)


def test_growing_cycle_overflows_the_stack(rq):
    # nodes 0 and 1 each have two children, nodes 0 and 1: the stack grows by one per visit
    node = cw_node(0, 0, 0x03, {0: INNER0, 1: INNER1}, [0, 1])
    scene = rq.Scene.from_arrays(rq.CWBVH, np.concatenate([node, node]), np.zeros((3, 4), np.float32))
    ctx = rq.Context()
    hits = _trace(rq, ctx, scene, rays_inside(256), rq.CLOSEST)
    with pytest.raises(rq.RQError, match="STACK_OVERFLOW"):
        ctx.check()
    assert (hits[:, 1].view(np.int32) == -1).all()
    _valid_after(rq, ctx)


@pytest.mark.parametrize("case", ["child", "triangle"])
def test_out_of_range_addresses(rq, case):
    if case == "child":
        nodes = cw_node(1000, 0, 0x01, {0: INNER0}, [0])  # child node 1000 of a 1-node buffer
    else:
        nodes = cw_node(0, 1000, 0x00, {0: LEAF1}, [0])   # triangle 1000 of a 1-triangle buffer
    scene = rq.Scene.from_arrays(rq.CWBVH, nodes, np.zeros((3, 4), np.float32))
    ctx = rq.Context()
    for query in (rq.CLOSEST, rq.ANY):
        hits = _trace(rq, ctx, scene, rays_inside(512), query)
        with pytest.raises(rq.RQError, match="BAD_SCENE"):
            ctx.check()
        assert (hits[:, 1].view(np.int32) == -1).all()
    _valid_after(rq, ctx)


@pytest.mark.parametrize("case", ["child", "unterminated_leaf"])
def test_bvh2_out_of_range(rq, case):
    n = np.zeros((4, 4), np.float32)
    box = [0.0, 255.0, 0.0, 255.0]
    n[0] = box
    n[1] = box
    n[2] = [0.0, 255.0, 0.0, 255.0]
    if case == "child":
        kids = np.array([400, 404, 0, 0], np.int32)  # node float4 indices far past the buffer
    else:
        kids = np.array([~0, ~0, 0, 0], np.int32)    # leaf at Woop row 0 with no terminator after it
    n[3] = kids.view(np.float32)
    woop = np.zeros((3, 4), np.float32)
    scene = rq.Scene.from_arrays(rq.BVH2, n, woop)
    ctx = rq.Context()
    hits = _trace(rq, ctx, scene, rays_inside(512), rq.CLOSEST)
    with pytest.raises(rq.RQError, match="BAD_SCENE"):
        ctx.check()
    assert (hits[:, 1].view(np.int32) == -1).all()
    _valid_after(rq, ctx)


def test_misaligned_buffers_refused(rq):
    """Ray and hit buffers are float4 records: a pointer off a 16-byte
    boundary is refused with RQ_ERR_INVALID_ARG before any launch."""
    import torch
    n = cw_node(1, 0, 0, {}, [])
    scene = rq.Scene.from_arrays(rq.CWBVH, n, np.zeros((3, 4), np.float32))
    ctx = rq.Context()
    raw = torch.zeros(64 * 8 + 4, dtype=torch.float32, device="cuda")
    hits = torch.zeros((64, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.trace(ctx, scene, raw[2:2 + 64 * 8].view(64, 8), hits, rq.ANY)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.trace(ctx, scene, raw[:64 * 8].view(64, 8), raw[2:2 + 64 * 4].view(64, 4), rq.ANY)
    _valid_after(rq, ctx)
