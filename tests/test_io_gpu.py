"""The reference's main() path end to end through files: mesh.dat ->
build + convert -> rtBindCWBVHData; samplecache.dat -> GenerateAORaysUniform
(32 rays per texel, src/main.cpp:66-78) -> rtTraceCWBVH / rtOccludedCWBVH,
checked against the oracle; and a scene reloaded from its scene file traces
bit-identically to the one it was saved from."""
import numpy as np
import pytest

from adjudicate import compare

pytestmark = pytest.mark.gpu


def _surfels(V, I, n, seed):
    rng = np.random.default_rng(seed)
    tri = rng.integers(0, I.shape[0], n)
    a, b = np.sqrt(rng.random(n)), rng.random(n)
    p0, p1, p2 = V[I[tri, 0]], V[I[tri, 1]], V[I[tri, 2]]
    P = p0 * (1 - a)[:, None] + p1 * (a * (1 - b))[:, None] + p2 * (a * b)[:, None]
    Nn = np.cross(p1 - p0, p2 - p0)
    Nn /= np.maximum(np.linalg.norm(Nn, axis=1, keepdims=True), 1e-30)
    pos = np.concatenate([P, np.ones((n, 1))], 1).astype(np.float32)
    nrm = np.concatenate([Nn, np.zeros((n, 1))], 1).astype(np.float32)
    return pos, nrm, np.full(n, 0.002, np.float32)


def test_reference_main_through_files(rq, po, tmp_path):
    import torch
    V, I = rq.gen_heightfield_boxes(11)
    rq.save_mesh_dat(tmp_path / "mesh.dat", V, I)
    sx, sy = 64, 48
    pos, nrm, rad = _surfels(V, I, sx * sy, 2)
    rq.save_samplecache_dat(tmp_path / "samplecache.dat", sx, sy, pos, nrm, rad)

    v, i, _ = rq.load_mesh_dat(tmp_path / "mesh.dat")
    hb = rq.HostBVH(v, i, rq.CWBVH)
    nodes = torch.from_numpy(hb.nodes).cuda()
    woop = torch.from_numpy(hb.woop).cuda()
    prim = torch.from_numpy(hb.prim_index).cuda()
    rq.rtBindCWBVHData(nodes, woop, prim)
    gx, gy, p, n, r = rq.load_samplecache_dat(tmp_path / "samplecache.dat")
    rays = rq.GenerateAORaysUniform(gx * gy, 32, p, n, r)
    count = gx * gy * 32
    assert rays.shape == (count, 8)
    hits = torch.empty((count, 4), device="cuda")
    rq.rtTraceCWBVH(rays, hits, count)
    rr = rays.cpu().numpy()
    want = po.trace(rq.CWBVH, hb.nodes, hb.woop, rr, False)
    compare(po, rr, hits.cpu().numpy(), want, hb.prim_index, v, i, any_hit=False)
    rq.rtOccludedCWBVH(rays, hits, count)
    wa = po.trace(rq.CWBVH, hb.nodes, hb.woop, rr, True)
    got = hits.cpu().numpy()[:, 1].view(np.int32) != -1
    assert np.array_equal(got, wa[:, 1].view(np.int32) != -1)
    assert 0.05 < got.mean() < 0.95


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_reloaded_scene_traces_identically(rq, tmp_path, kind):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = rq.gen_heightfield_boxes(4)
    ds = W.upload(V, I, kind)
    ds.host.save(tmp_path / "s.rqs")
    sc2 = rq.Scene.from_host(rq.HostBVH.load(tmp_path / "s.rqs"))
    rays = W.ao_rays(ds, 100_000, seed=9)
    ctx = rq.Context()
    for q in (rq.CLOSEST, rq.ANY):
        a = torch.empty((rays.shape[0], 4), device="cuda")
        b = torch.empty_like(a)
        rq.trace_ordered(ctx, ds.scene, rays, a, q)
        rq.trace_ordered(ctx, sc2, rays, b, q)
        ctx.check()
        assert torch.equal(a.view(torch.int32), b.view(torch.int32))
