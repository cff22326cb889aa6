"""Parity at the benchmark workloads' full sizes.

The oracle traces only small ray sets in seconds, so at full size every ray
is checked through properties that hold at any size, and a seeded sample of
rays is traced by the oracle on the full trees:

* any-hit occlusion bits equal closest-hit hit flags, bit for bit: a closest
  hit exists exactly when some triangle lies in the ray's interval, and the
  Woop test of a (ray, triangle) pair does not depend on the schedule;
* the batch equals per-scene launches, Morton-sorted equals unsorted, and the
  fused AO counts equal the reduction of the hit buffer (occlusion bits);
* the ordered kernel's output for the sampled rays equals the oracle bit for
  bit (a ray's traversal order there does not depend on the other rays of
  the launch), and the production kernel's closest primitive ids agree with
  the oracle's, every disagreement adjudicated in FP64 (tests/adjudicate.py).

Workloads: the 29.6M-triangle spheres-and-terrain scene with 16M surfels x 4
AO rays, the 64-scene batch (19.1M triangles, 126.7M AO rays), and the 0.95M
triangle city with 4096 x 4096 camera rays in 4 x 8 tiles.
"""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from adjudicate import compare

pytestmark = pytest.mark.gpu

SAMPLE = 4096


def _hit_flags(hits):
    import torch
    return hits[:, 1].view(torch.int32) != -1


def _sample(n: int, k: int, seed: int) -> np.ndarray:
    return np.sort(np.random.default_rng(seed).choice(n, size=min(k, n), replace=False))


def _check_sample(rq, po, ctx, ds, V, I, rays, idx, query, prod_hits):
    """Ordered kernel over the full ray set, bit-exact on the sampled rays;
    the production hits of the sampled rays adjudicated against the oracle."""
    import torch
    ordered = torch.empty((rays.shape[0], 4), device="cuda")
    rq.trace_ordered(ctx, ds.scene, rays, ordered, query)
    ctx.check()
    t_idx = torch.from_numpy(idx).cuda()
    r = rays[t_idx].cpu().numpy()
    want = po.trace(rq.CWBVH, ds.host.nodes, ds.host.woop, r, query == rq.ANY)
    got_ordered = ordered[t_idx].cpu().numpy()
    compare(po, r, got_ordered, want, ds.host.prim_index, V, I, query == rq.ANY, exact=True)
    return compare(po, r, prod_hits[t_idx].cpu().numpy(), want, ds.host.prim_index, V, I, query == rq.ANY)


@pytest.fixture(scope="module")
def large(rq):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = rq.gen_spheres_terrain(0, 30_000_000)
    ds = W.upload(V, I, rq.CWBVH)
    rays = W.ao_rays(ds, 1 << 26, seed=2000, spp=4)
    torch.cuda.synchronize()
    return V, I, ds, rays


def test_large_scene_full_size(rq, po, large):
    import torch
    V, I, ds, rays = large
    assert I.shape[0] > 29_000_000 and rays.shape[0] == 1 << 26
    ctx = rq.Context()
    n = rays.shape[0]
    any_h = torch.empty((n, 4), device="cuda")
    clo_h = torch.empty((n, 4), device="cuda")
    rq.trace(ctx, ds.scene, rays, any_h, rq.ANY)
    rq.trace(ctx, ds.scene, rays, clo_h, rq.CLOSEST)
    ctx.check()
    occ = _hit_flags(any_h)
    assert torch.equal(occ, _hit_flags(clo_h))
    assert 0.05 < occ.float().mean().item() < 0.95

    # Morton-sorted inside a one-item batch, hits scattered back to ray order.
    sorted_h = torch.empty((n, 4), device="cuda")
    b = rq.Batch(ctx, [(ds.scene, rays, sorted_h)], rq.ANY, sort_threshold=0)
    b.run()
    torch.cuda.synchronize()
    ctx.check()
    b.close()
    assert torch.equal(occ, _hit_flags(sorted_h))
    del sorted_h

    # Fused AO counts (no hit buffer) equal the per-surfel sum of the bits.
    counts = rq.trace_ao(ctx, ds.scene, rays, 4)
    ctx.check()
    assert torch.equal(counts, occ.view(-1, 4).sum(1, dtype=torch.int32))

    idx = _sample(n, SAMPLE, 1)
    res = _check_sample(rq, po, ctx, ds, V, I, rays, idx, rq.ANY, any_h)
    assert res["hits"] > SAMPLE // 20
    _check_sample(rq, po, ctx, ds, V, I, rays, idx, rq.CLOSEST, clo_h)


@pytest.fixture(scope="module")
def batched(rq):
    import torch
    from cwbvh_b200 import workloads as W
    tris, counts = W.batched_sizes(64)

    def build(i):
        V, I = W.scene_of_size(i, int(tris[i]))
        return V, I, rq.HostBVH(V, I, rq.CWBVH, threads=1)

    with cf.ThreadPoolExecutor(max_workers=max(1, min(64, os.cpu_count() or 1))) as ex:
        built = list(ex.map(build, range(64)))
    out = []
    for i, (V, I, hb) in enumerate(built):
        ds = W.DeviceScene(rq.CWBVH, hb, rq.Scene.from_host(hb), torch.from_numpy(V).cuda(),
                           torch.from_numpy(I).cuda(), W.diag(V), I.shape[0])
        out.append((V, I, ds, W.ao_rays(ds, int(counts[i]), seed=i + 1000)))
    torch.cuda.synchronize()
    return out


def test_batched_workload_full_size(rq, po, batched):
    import torch
    assert sum(r.shape[0] for *_, r in batched) > 126_000_000
    ctx = rq.Context()
    any_b = [torch.empty((r.shape[0], 4), device="cuda") for *_, r in batched]
    clo_b = [torch.empty((r.shape[0], 4), device="cuda") for *_, r in batched]
    for query, hits in ((rq.ANY, any_b), (rq.CLOSEST, clo_b)):
        b = rq.Batch(ctx, [(ds.scene, r, h) for (_, _, ds, r), h in zip(batched, hits)], query, use_graph=True)
        b.run()
        b.run()  # graph replay after the capture run
        torch.cuda.synchronize()
        ctx.check()
        b.close()
    plain = torch.empty((max(r.shape[0] for *_, r in batched), 4), device="cuda")
    for k, (V, I, ds, r) in enumerate(batched):
        occ = _hit_flags(any_b[k])
        assert torch.equal(occ, _hit_flags(clo_b[k])), f"scene {k}"
        p = plain[: r.shape[0]]
        rq.trace(ctx, ds.scene, r, p, rq.ANY)
        ctx.check()
        assert torch.equal(occ, _hit_flags(p)), f"scene {k}"
    # Sampled oracle parity on the smallest, the largest and six other scenes.
    n_tris = [ds.n_tris for _, _, ds, _ in batched]
    picks = sorted({int(np.argmin(n_tris)), int(np.argmax(n_tris))} | set(range(0, 64, 11)))
    for k in picks:
        V, I, ds, r = batched[k]
        idx = _sample(r.shape[0], 1024, k)
        _check_sample(rq, po, ctx, ds, V, I, r, idx, rq.ANY, any_b[k])
        _check_sample(rq, po, ctx, ds, V, I, r, idx, rq.CLOSEST, clo_b[k])


def test_city_full_size(rq, po):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = rq.gen_city(0, 10000)
    ds = W.upload(V, I, rq.CWBVH)
    dg = W.diag(V)
    lo, hi = V.min(0), V.max(0)
    ext = hi - lo
    eye = (float(lo[0] - 0.05 * ext[0]), float(lo[1] - 0.05 * ext[1]), float(0.25 * max(ext[0], ext[1])))
    look = (float(0.5 * (lo[0] + hi[0])), float(0.5 * (lo[1] + hi[1])), 0.0)
    prim = rq.camera_rays(eye, look, (0.0, 0.0, 1.0), 60.0, 4096, 4096, 0.0, 10.0 * dg, tile=(4, 8))
    n = prim.shape[0]
    ctx = rq.Context()
    ph = torch.empty((n, 4), device="cuda")
    rq.trace(ctx, ds.scene, prim, ph, rq.CLOSEST)
    ctx.check()
    assert 0.5 < _hit_flags(ph).float().mean().item() < 1.0
    _check_sample(rq, po, ctx, ds, V, I, prim, _sample(n, SAMPLE, 2), rq.CLOSEST, ph)

    pos, nrm, rad = rq.surfels_from_hits(prim, ph, ds.scene)
    ao = rq.aorays(pos, nrm, rad, 1, seed=77, tmin=1e-4 * dg, tmax=0.05 * dg, offset_scale=0.0)
    del pos, nrm, rad
    ah = torch.empty((n, 4), device="cuda")
    ch = torch.empty((n, 4), device="cuda")
    rq.trace(ctx, ds.scene, ao, ah, rq.ANY)
    rq.trace(ctx, ds.scene, ao, ch, rq.CLOSEST)
    ctx.check()
    assert torch.equal(_hit_flags(ah), _hit_flags(ch))
    # Rays of pixels that missed are empty intervals and never hit.
    assert not (_hit_flags(ah) & ~_hit_flags(ph)).any()
    _check_sample(rq, po, ctx, ds, V, I, ao, _sample(n, SAMPLE, 3), rq.ANY, ah)
