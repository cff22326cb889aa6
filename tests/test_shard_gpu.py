"""One ray set over several devices holding replicas of one scene
(rq_sharded_*): contiguous ray ranges per device, hits gathered into the
caller's buffer by peer copies.  The tests here have one GPU, so the parts
repeat device 0 (each part still has its own context, stream and staging
buffers, and the copies run as on distinct devices); the gathered hits must
equal one trace of the whole buffer bit for bit, on ragged counts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", [0, 1])
def test_sharded_equals_one_trace(rq, kind):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    # the oracle's traversal order, so a ray's result does not depend on its warp
    launch = rq.default_launch(kind, rq.ANY)
    launch.postpone_ratio = -1.0
    scenes = [W.upload(V, I, kind) for _ in range(3)]
    rays_all = W.ao_rays(scenes[0], 1_000_003, seed=1000)
    ctx = rq.Context()
    for parts in (1, 2, 3):
        sh = rq.Sharded([0] * parts, [ds.scene for ds in scenes[:parts]], max_rays=rays_all.shape[0])
        for n in (1_000_003, 2, 0):
            rays = rays_all[:n].contiguous()
            for q in (rq.ANY, rq.CLOSEST):
                got = torch.full((n, 4), float("nan"), device="cuda")
                sh.trace(rays, got, q, launch=launch)
                want = torch.empty((n, 4), device="cuda")
                if n:
                    rq.trace(ctx, scenes[0].scene, rays, want, q, launch=launch)
                ctx.check()
                g, w = got.cpu().numpy(), want.cpu().numpy()
                assert np.array_equal(g[:, 1].view(np.int32) != -1, w[:, 1].view(np.int32) != -1)
                if q == rq.CLOSEST:
                    # the closest t is unique; BVH2's speculative schedule may
                    # pick another of several triangles at exactly that t
                    assert np.array_equal(g[:, 0].view(np.uint32), w[:, 0].view(np.uint32))
                    if kind == rq.CWBVH:
                        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
        sh.close()


def test_sharded_refuses_more_rays_than_created_for(rq):
    import torch
    from cwbvh_b200 import workloads as W
    ds = W.upload(*W.heightfield_boxes(0), rq.CWBVH)
    sh = rq.Sharded([0, 0], [ds.scene, ds.scene], max_rays=100)
    rays = W.ao_rays(ds, 101, seed=7)
    hits = torch.empty((101, 4), device="cuda")
    with pytest.raises(rq.RQError):
        sh.trace(rays, hits, rq.ANY)
    assert "100" in rq.lib.rq_last_error().decode()
    sh.trace(rays[:100].contiguous(), hits[:100], rq.ANY)
    sh.close()
