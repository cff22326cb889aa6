"""Primary visibility + ambient occlusion over the city scene, stage by stage
on the GPU against the oracle: pinhole camera rays -> closest hit ->
surfels at the hit points -> AO rays -> any-hit -> per-surfel AO.

Each stage's input is the GPU's own output of the stage before it, so the
trace stages are compared on identical rays (bit-exact for the ordered
kernel, adjudicated for the production schedule) and the generators within
float tolerance of a numpy / oracle restatement.
"""
import numpy as np
import pytest

from adjudicate import compare

pytestmark = pytest.mark.gpu

W_PX, H_PX, SPP = 192, 128, 4
EYE, LOOK, UP = (-60.0, -40.0, 140.0), (200.0, 220.0, 0.0), (0.0, 0.0, 1.0)


@pytest.fixture(scope="module")
def city(rq):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = rq.gen_city(seed=7, n_buildings=400)
    ds = W.upload(V, I, rq.CWBVH)
    torch.cuda.synchronize()
    return V, I, ds


def _camera_numpy(w, h, vfov):
    e, l, u = (np.array(x, np.float64) for x in (EYE, LOOK, UP))
    f = (l - e) / np.linalg.norm(l - e)
    r = np.cross(f, u)
    r /= np.linalg.norm(r)
    up = np.cross(r, f)
    hh = np.tan(np.radians(vfov) / 2)
    hw = hh * w / h
    x, y = np.meshgrid(np.arange(w), np.arange(h))
    sx = ((x.ravel() + 0.5) / w * 2 - 1) * hw
    sy = (1 - (y.ravel() + 0.5) / h * 2) * hh
    d = f[None] + sx[:, None] * r[None] + sy[:, None] * up[None]
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def test_camera_rays(rq):
    rays = rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tmin=0.0, tmax=1e4).cpu().numpy()
    assert rays.shape == (W_PX * H_PX, 8)
    assert np.array_equal(rays[:, 0:3], np.tile(np.array(EYE, np.float32), (W_PX * H_PX, 1)))
    assert (rays[:, 3] == 0).all() and (rays[:, 7] == np.float32(1e4)).all()
    assert np.abs(rays[:, 4:7] - _camera_numpy(W_PX, H_PX, 50.0)).max() < 2e-6


def test_camera_rays_tiled(rq):
    """Tile order is a permutation of the row-major rays, bit for bit."""
    import torch
    rows = rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tmin=0.0, tmax=1e4)
    tw, th = 4, 8
    tiled = rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tmin=0.0, tmax=1e4, tile=(tw, th))
    i = np.arange(W_PX * H_PX)
    tile, r = i // (tw * th), i % (tw * th)
    x = (tile % (W_PX // tw)) * tw + r % tw
    y = (tile // (W_PX // tw)) * th + r // tw
    pix = torch.from_numpy(y * W_PX + x).cuda()
    assert torch.equal(tiled.view(torch.int32), rows[pix].view(torch.int32))
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tile=(5, 8))  # 192 is not a multiple of 5
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tile=(0, 8))


def test_camera_rays_bad_args(rq):
    with pytest.raises(rq.RQError):
        rq.camera_rays(EYE, EYE, UP, 50.0, 8, 8)  # look == eye
    with pytest.raises(rq.RQError):
        rq.camera_rays(EYE, LOOK, UP, 0.0, 8, 8)


@pytest.mark.parametrize("ordered", [True, False], ids=["ordered", "production"])
def test_city_primary_and_ao(rq, po, city, ordered):
    import torch
    V, I, ds = city
    ctx = rq.Context()
    trace = rq.trace_ordered if ordered else rq.trace
    host = ds.host

    rays = rq.camera_rays(EYE, LOOK, UP, 50.0, W_PX, H_PX, tmin=0.0, tmax=1e4)
    hits = torch.full((rays.shape[0], 4), float("nan"), device="cuda")
    trace(ctx, ds.scene, rays, hits, rq.CLOSEST)
    ctx.check()
    r, g = rays.cpu().numpy(), hits.cpu().numpy()
    want = po.trace(rq.CWBVH, host.nodes, host.woop, r, False)
    res = compare(po, r, g, want, host.prim_index, V, I, False, exact=ordered)
    ids = g[:, 1].view(np.int32)
    assert 0.5 < (ids >= 0).mean() < 1.0  # ground, facades and some sky

    # Surfels: hit point o + t d and the facing unit normal of the hit triangle.
    pos, nrm, rad = rq.surfels_from_hits(rays, hits, ds.scene)
    p, n = pos.cpu().numpy(), nrm.cpu().numpy()
    hit = ids >= 0
    assert np.allclose(p[hit, :3], r[hit, :3] + g[hit, 0:1] * r[hit, 4:7], rtol=0, atol=1e-3)
    assert np.array_equal(p[~hit, :3], r[~hit, :3]) and (n[~hit] == 0).all()
    assert np.allclose(np.linalg.norm(n[hit, :3], axis=1), 1, atol=1e-5)
    assert (np.einsum("ij,ij->i", n[hit, :3], r[hit, 4:7]) <= 0).all()
    # Ground hits (z ~ 0) face straight up.
    ground = hit & (np.abs(p[:, 2]) < 1e-3) & (np.abs(n[:, 2]) > 0.5)
    assert ground.sum() > 100 and np.allclose(n[ground, :3], [0, 0, 1], atol=1e-6)

    # AO rays from those surfels, then any-hit.
    ao_rays = rq.aorays(pos, nrm, rad, SPP, seed=11, tmin=1e-3, tmax=30.0, offset_scale=0.0)
    ar = ao_rays.cpu().numpy()
    want_rays = po.aorays(p, n, rad.cpu().numpy(), SPP, 11, 1e-3, 30.0, 0.0)
    assert np.abs(ar[:, 4:7] - want_rays[:, 4:7]).max() < 1e-4  # sinf/cosf: device vs libm ulps
    miss_rows = np.repeat(~hit, SPP)
    assert (ar[miss_rows, 7] == 0).all() and np.array_equal(ar[miss_rows], want_rays[miss_rows])
    ao_hits = torch.full((ao_rays.shape[0], 4), float("nan"), device="cuda")
    trace(ctx, ds.scene, ao_rays, ao_hits, rq.ANY)
    ctx.check()
    ag = ao_hits.cpu().numpy()
    want_ao = po.trace(rq.CWBVH, host.nodes, host.woop, ar, True)
    compare(po, ar, ag, want_ao, host.prim_index, V, I, True, exact=ordered)
    assert (ag[miss_rows, 1].view(np.int32) == -1).all()

    ao = rq.ao_reduce(ao_hits, rays.shape[0], SPP).cpu().numpy()
    occ = (want_ao[:, 1].view(np.int32) != -1).reshape(-1, SPP).mean(axis=1)
    if ordered:
        assert np.array_equal(ao, occ.astype(np.float32))
    else:
        assert np.abs(ao - occ).max() <= 1.0 / SPP and (ao != occ).mean() < 1e-3
    assert 0.05 < ao[hit].mean() < 0.95
    assert res["hits"] > 0
