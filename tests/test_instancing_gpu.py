"""Two-level traversal on the GPU (rq_trace_instanced) against the oracle's
instanced traversal on the same top-level buffers: bit-identical hits and
the same instance per ray; the semantics against the flattened mesh are
covered on the CPU (test_instancing.py)."""
import numpy as np
import pytest

from instancing_common import make_instances, world_rays

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu_inst(rq):
    meshes, blas, M, bi, flat, tri_off = make_instances(rq, n_inst=2000, seed=4)
    scenes = [rq.Scene.from_host(b) for b in blas]
    tlas = rq.Tlas(scenes, M, bi)
    return blas, scenes, tlas, M, bi


@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_instanced_kernel_bit_exact(rq, po, gpu_inst, query):
    import torch
    blas, scenes, tlas, M, bi = gpu_inst
    rays = world_rays(200_000, 11)
    r = torch.from_numpy(rays).cuda()
    hits = torch.full((rays.shape[0], 4), float("nan"), device="cuda")
    inst = torch.full((rays.shape[0],), -7, dtype=torch.int32, device="cuda")
    ctx = rq.Context()
    rq.trace_instanced(ctx, tlas, r, hits, query, instance_out=inst, ordered=True)
    ctx.check()
    want, wi = po.trace_instanced(tlas.buffers(), [(b.nodes, b.woop) for b in blas], rays, query == rq.ANY)
    got = hits.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(inst.cpu().numpy(), wi)
    hit = want[:, 1].view(np.int32) >= 0
    assert 0.1 < hit.mean() < 0.9
    assert (wi[hit] >= 0).all() and (wi[~hit] == -1).all()


@pytest.mark.parametrize("query", [0, 1], ids=["closest", "any"])
def test_instanced_postponing_schedule(rq, po, gpu_inst, query):
    """With triangle / instance postponing the order changes: occlusion must
    be identical, closest hits identical except exact ties in t."""
    import torch
    blas, scenes, tlas, M, bi = gpu_inst
    rays = world_rays(200_000, 12)
    r = torch.from_numpy(rays).cuda()
    hits = torch.empty((rays.shape[0], 4), device="cuda")
    inst = torch.empty((rays.shape[0],), dtype=torch.int32, device="cuda")
    ctx = rq.Context()
    rq.trace_instanced(ctx, tlas, r, hits, query, instance_out=inst, launch=rq.Launch(0, 0, 0, 0.2, 0, 0))
    ctx.check()
    want, wi = po.trace_instanced(tlas.buffers(), [(b.nodes, b.woop) for b in blas], rays, query == rq.ANY)
    got, gi = hits.cpu().numpy(), inst.cpu().numpy()
    g_hit, w_hit = got[:, 1].view(np.int32) >= 0, want[:, 1].view(np.int32) >= 0
    assert np.array_equal(g_hit, w_hit)
    if query == rq.CLOSEST:
        diff = (got[:, 1].view(np.int32) != want[:, 1].view(np.int32)) | (gi != wi)
        # the closest t does not depend on the order up to ties within
        # rounding; only such ties may pick the other triangle
        assert np.allclose(got[:, 0], want[:, 0], rtol=1e-6, atol=0)
        assert diff.mean() < 1e-4, diff.sum()


def test_tlas_validation(rq, gpu_inst):
    from cwbvh_b200 import workloads as W
    blas, scenes, tlas, M, bi = gpu_inst
    V, I = rq.gen_heightfield_boxes(0, grid=8, n_boxes=2)
    b2 = W.upload(V, I, rq.BVH2)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.Tlas([b2.scene], M[:1], np.zeros(1, np.int32))
    bad = M[:4].copy()
    bad[1] = 0
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.Tlas(scenes, bad, bi[:4])
    one = rq.Tlas(scenes[:1], np.eye(3, 4, dtype=np.float32)[None], np.zeros(1, np.int32))
    assert one.n_instances == 1
    one.close()
