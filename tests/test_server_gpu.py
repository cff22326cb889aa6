"""Continuous-batching server: every request's result is the same alone and in
the mix; requests arriving while others run are admitted and overlap; failures
(unknown scene, over-budget request, cancellation, shutdown) come back as
status codes."""
import threading

import numpy as np
import pytest

from adjudicate import prim_ids

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes(rq):
    import torch
    from cwbvh_b200 import workloads as W
    out = []
    for seed, tris in ((0, 20000), (1, 60000), (2, 5000)):
        V, I = W.scene_of_size(seed, tris)
        ds = W.upload(V, I, rq.CWBVH)
        out.append(ds)
    torch.cuda.synchronize()
    return out


def _rays(W, ds, n, seed):
    return W.ao_rays(ds, n, seed=seed).cpu().numpy()


def _pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()


def test_results_same_alone_and_in_mix(rq, scenes):
    from cwbvh_b200 import workloads as W
    rng = np.random.default_rng(0)
    reqs = []
    for k in range(24):
        sid = int(rng.integers(0, len(scenes)))
        n = int(np.exp(rng.uniform(np.log(4000), np.log(200_000))))
        rays = _pinned((n, 8))
        rays[:] = _rays(W, scenes[sid], n, 100 + k)
        reqs.append((sid, rays))
    # alone: one request at a time
    alone = []
    srv = rq.Server(hbm_budget_bytes=1 << 30, query=rq.ANY, streams=3)
    ids = [srv.add_scene(ds.scene) for ds in scenes]
    for sid, rays in reqs:
        hits = _pinned((rays.shape[0], 4))
        t = srv.submit(ids[sid], rays, hits)
        st = srv.wait(t)
        assert st["status"] == 0
        alone.append(hits.copy())
    # in the mix: the server's three streams are first kept busy by large
    # requests (pageable hit buffers: their results come back after the
    # stream's work), then all requests are submitted at once from two
    # threads, pageable and pinned buffers, while those run
    big = 3_000_000
    blockers = []
    for k in range(3):
        br = _pinned((big, 8))
        br[:] = _rays(W, scenes[1], big, 900 + k)
        bh = np.zeros((big, 4), np.float32)
        blockers.append((br, bh, srv.submit(ids[1], br, bh)))
    mix = [None] * len(reqs)
    tickets = [None] * len(reqs)

    def submitter(ks):
        for k in ks:
            sid, rays = reqs[k]
            hits = np.zeros((rays.shape[0], 4), np.float32) if k % 2 else _pinned((rays.shape[0], 4))
            mix[k] = hits
            tickets[k] = srv.submit(ids[sid], rays, hits)

    th = [threading.Thread(target=submitter, args=(range(j, len(reqs), 2),)) for j in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    stats = [srv.wait(t) for t in tickets]
    for _, _, t in blockers:
        assert srv.wait(t)["status"] == 0
    srv.close()
    batches = {s["batch_id"] for s in stats}
    assert len(batches) < len(reqs)  # requests that arrived while others ran shared launches
    for k, (sid, rays) in enumerate(reqs):
        pi = scenes[sid].host.prim_index
        assert np.array_equal(prim_ids(alone[k], pi) >= 0, prim_ids(mix[k], pi) >= 0), k
    lat = np.array([s["done_ms"] - s["submit_ms"] for s in stats])
    assert np.isfinite(np.percentile(lat, 99))


def test_results_match_plain_trace(rq, scenes):
    import torch
    from cwbvh_b200 import workloads as W
    srv = rq.Server(hbm_budget_bytes=256 << 20, query=rq.ANY, streams=2)
    sid = srv.add_scene(scenes[1].scene)
    rays = _pinned((100_000, 8))
    rays[:] = _rays(W, scenes[1], 100_000, 7)
    hits = _pinned((100_000, 4))
    srv.wait(srv.submit(sid, rays, hits))
    srv.close()
    ctx = rq.Context()
    h = torch.empty((100_000, 4), device="cuda")
    rq.trace(ctx, scenes[1].scene, torch.from_numpy(rays).cuda(), h, rq.ANY)
    ctx.check()
    pi = scenes[1].host.prim_index
    assert np.array_equal(prim_ids(hits, pi) >= 0, prim_ids(h.cpu().numpy(), pi) >= 0)


def test_failures_are_status_codes(rq, scenes):
    from cwbvh_b200 import workloads as W
    srv = rq.Server(hbm_budget_bytes=48 * 3 * 50_000, query=rq.ANY, streams=3)  # 50k rays per launch
    sid = srv.add_scene(scenes[0].scene)
    rays = _pinned((60_000, 8))
    rays[:] = _rays(W, scenes[0], 60_000, 9)
    hits = _pinned((60_000, 4))
    with pytest.raises(rq.RQError) as e:
        srv.submit(99, rays[:10], hits[:10])
    assert e.value.status == 7  # RQ_ERR_NOT_FOUND
    with pytest.raises(rq.RQError) as e:
        srv.wait(123456)
    assert e.value.status == 7
    # Queue more than the pool can hold; cancel the last queued one.
    tickets = [srv.submit(sid, rays[:40_000], hits[:40_000]) for _ in range(8)]
    cancelled = srv.cancel(tickets[-1])
    for t in tickets[:-1]:
        assert srv.wait(t)["status"] == 0
    if cancelled == 0:
        with pytest.raises(rq.RQError) as e:
            srv.wait(tickets[-1])
        assert e.value.status == 9  # RQ_ERR_CANCELLED
    srv.close()


def test_budget_binds_and_large_requests_are_split(rq, scenes):
    """A pool that holds about two launches: requests queue for bytes, the
    bytes in use never exceed the budget, requests larger than one launch are
    cut into pieces, and every result equals one plain trace of its rays."""
    import torch
    from cwbvh_b200 import workloads as W
    per_launch = 30_000
    budget = 2 * (per_launch * 48 + 512) + 256
    srv = rq.Server(hbm_budget_bytes=budget, query=rq.ANY, streams=3, max_batch_rays=per_launch)
    ids = [srv.add_scene(ds.scene) for ds in scenes]
    rng = np.random.default_rng(5)
    reqs = []
    for k in range(14):
        sid = k % len(scenes)
        n = int(rng.integers(1000, 100_000)) if k % 3 else 95_001  # some span several launches
        rays = _pinned((n, 8))
        rays[:] = _rays(W, scenes[sid], n, 700 + k)
        reqs.append((sid, rays, np.zeros((n, 4), np.float32) if k % 2 else _pinned((n, 4))))
    tickets = [srv.submit(ids[sid], r, h) for sid, r, h in reqs]
    stats = [srv.wait(t) for t in tickets]
    mem = srv.memory()
    srv.close()
    assert all(s["status"] == 0 for s in stats)
    assert mem["pool_bytes"] == budget // 256 * 256
    assert 0 < mem["peak_in_use_bytes"] <= mem["pool_bytes"]
    assert mem["admission_waits"] > 0  # the budget, not the streams, held requests back
    assert mem["pieces"] == sum(-(-r.shape[0] // per_launch) for _, r, _ in reqs)
    ctx = rq.Context()
    for sid, rays, hits in reqs:
        h = torch.empty((rays.shape[0], 4), device="cuda")
        rq.trace(ctx, scenes[sid].scene, torch.from_numpy(rays).cuda(), h, rq.ANY)
        ctx.check()
        pi = scenes[sid].host.prim_index
        assert np.array_equal(prim_ids(hits, pi) >= 0, prim_ids(h.cpu().numpy(), pi) >= 0)


def _surfels(rq, ds, n, seed):
    pos, nrm, rad = rq.sample_surfels(ds.vertices, ds.indices, n, seed)
    rad.fill_(0.001)
    return pos.cpu().numpy(), nrm.cpu().numpy(), rad.cpu().numpy()


def test_bake_requests_equal_trace_then_reduce(rq, scenes):
    """A bake request (surfels in, AO out; rays generated and counted on the
    device) gives exactly rq_aorays + rq_trace any-hit + rq_ao_reduce, alone
    and mixed with ray requests in the same batches."""
    import torch
    from cwbvh_b200 import workloads as W
    srv = rq.Server(hbm_budget_bytes=1 << 30, query=rq.ANY, streams=2)
    ids = [srv.add_scene(ds.scene) for ds in scenes]
    ctx = rq.Context()
    jobs = []
    for k in range(9):
        sid, spp = k % len(scenes), (1, 8, 32)[k % 3]
        n = 3000 + 1500 * k
        pos, nrm, rad = _surfels(rq, scenes[sid], n, 40 + k)
        rad = rad if k % 4 else None  # radius-less requests too
        dg = scenes[sid].diag
        args = (spp, 500 + k, 1e-4 * dg, 0.1 * dg, 0.5)
        rays = rq.aorays(torch.from_numpy(pos).cuda(), torch.from_numpy(nrm).cuda(),
                         torch.from_numpy(rad).cuda() if rad is not None else None,
                         spp, seed=args[1], tmin=args[2], tmax=args[3], offset_scale=args[4])
        hits = torch.empty((rays.shape[0], 4), device="cuda")
        rq.trace(ctx, scenes[sid].scene, rays, hits, rq.ANY)
        want = rq.ao_reduce(hits, n, spp).cpu().numpy()
        ao = _pinned((n,)) if k % 2 else np.zeros(n, np.float32)  # pinned and pageable results
        jobs.append((sid, pos, nrm, rad, args, ao, want, n))
    ctx.check()
    mixed_rays = [(k % len(scenes), _pinned((20000, 8))) for k in range(4)]
    for k, (sid, r) in enumerate(mixed_rays):
        r[:] = _rays(W, scenes[sid], 20000, 900 + k)
    tickets = []
    for j, (sid, pos, nrm, rad, args, ao, want, n) in enumerate(jobs):
        tickets.append(srv.submit_bake(ids[sid], pos, nrm, rad, *args, ao))
        if j < len(mixed_rays):
            sid2, r = mixed_rays[j]
            tickets.append(srv.submit(ids[sid2], r, _pinned((20000, 4))))
    stats = [srv.wait(t) for t in tickets]
    assert all(s["status"] == 0 for s in stats)
    for sid, pos, nrm, rad, args, ao, want, n in jobs:
        assert np.array_equal(ao, want)
    assert any(0.0 < float(j[5].mean()) < 1.0 for j in jobs)
    srv.close()


def test_bake_request_errors(rq, scenes):
    pos = np.zeros((10, 4), np.float32)
    ao = np.zeros(10, np.float32)
    closest = rq.Server(hbm_budget_bytes=1 << 26, query=rq.CLOSEST)
    cid = closest.add_scene(scenes[0].scene)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        closest.submit_bake(cid, pos, pos, None, 4, 0, 0.0, 1.0, 0.0, ao)
    closest.close()
    small = rq.Server(hbm_budget_bytes=48 * 3000, query=rq.ANY, streams=1)
    sid = small.add_scene(scenes[0].scene)
    big = np.zeros((200, 4), np.float32)
    # one surfel's 4096 rays exceed a launch of this pool
    with pytest.raises(rq.RQError, match="BUDGET"):
        small.submit_bake(sid, big, big, None, 4096, 0, 0.0, 1.0, 0.0, np.zeros(200, np.float32))
    small.close()


def test_bake_request_split_into_pieces(rq, scenes):
    """A bake request larger than one launch is cut into whole-surfel pieces
    whose rays are generated with their indices in the whole request: the AO
    equals rq_aorays + rq_trace + rq_ao_reduce over all of it."""
    import torch
    ds = scenes[1]
    n, spp = 20_000, 16
    pos, nrm, rad = _surfels(rq, ds, n, 77)
    dg = ds.diag
    args = (spp, 4321, 1e-4 * dg, 0.1 * dg, 0.5)
    ctx = rq.Context()
    rays = rq.aorays(torch.from_numpy(pos).cuda(), torch.from_numpy(nrm).cuda(), torch.from_numpy(rad).cuda(), spp,
                     seed=args[1], tmin=args[2], tmax=args[3], offset_scale=args[4])
    hits = torch.empty((rays.shape[0], 4), device="cuda")
    rq.trace(ctx, ds.scene, rays, hits, rq.ANY)
    ctx.check()
    want = rq.ao_reduce(hits, n, spp).cpu().numpy()
    srv = rq.Server(hbm_budget_bytes=8 << 20, query=rq.ANY, streams=2, max_batch_rays=50_000)
    sid = srv.add_scene(ds.scene)
    ao = _pinned((n,))
    srv.wait(srv.submit_bake(sid, pos, nrm, rad, *args, ao))
    mem = srv.memory()
    srv.close()
    assert mem["pieces"] > 1
    assert np.array_equal(ao, want)
