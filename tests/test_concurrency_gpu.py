"""Scenes are immutable and every call is stream-ordered, so host threads
with their own contexts and streams may trace the same and different scenes
at the same time: results must equal the sequential ones, bit for bit for
occlusion and closest hits (the production schedule can reorder work within
a launch, but not across calls)."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_threads_and_streams_trace_concurrently(rq):
    import torch
    from cwbvh_b200 import workloads as W
    scenes = [W.upload(*W.heightfield_boxes(s), kind) for s, kind in ((0, rq.CWBVH), (1, rq.CWBVH), (2, rq.BVH2))]
    rays = [W.ao_rays(ds, 300_000, seed=50 + i) for i, ds in enumerate(scenes)]
    torch.cuda.synchronize()
    ctx0 = rq.Context()
    want = {}
    for i, (ds, r) in enumerate(zip(scenes, rays)):
        for q in (rq.ANY, rq.CLOSEST):
            h = torch.empty((r.shape[0], 4), device="cuda")
            rq.trace_ordered(ctx0, ds.scene, r, h, q)
            want[i, q] = h.cpu().numpy()
    ctx0.check()

    errors = []

    def worker(tid):
        try:
            ctx = rq.Context()
            stream = torch.cuda.Stream()
            for it in range(6):
                i = (tid + it) % len(scenes)
                q = rq.ANY if (tid + it) % 2 else rq.CLOSEST
                with torch.cuda.stream(stream):
                    h = torch.empty((rays[i].shape[0], 4), device="cuda")
                rq.trace_ordered(ctx, scenes[i].scene, rays[i], h, q, stream=stream)
                ctx.check(stream)
                stream.synchronize()
                g = h.cpu().numpy()
                if not np.array_equal(g.view(np.uint32), want[i, q].view(np.uint32)):
                    errors.append((tid, it, i, q))
        except Exception as e:  # pragma: no cover - reported below
            errors.append((tid, repr(e)))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
