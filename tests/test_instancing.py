"""Two-level scenes on the CPU: the top-level tree built on the host, and
the oracle's instanced traversal against the flattened world mesh (each
instance's triangles transformed to world space) -- the same occlusion and
closest triangles, every disagreement explained in FP64 on the world
triangles.  t is checked against the FP64 t of the same world triangle:
within 1e-4 relative plus 1e-6 / cos(angle of incidence) absolute (the ray
is transformed into object space in float; world coordinates reach 5, where
a float ulp is 5e-7, and grazing hits divide that by the cosine -- the
flattened mesh's own t carries errors of the same size)."""
import numpy as np
import pytest

from adjudicate import _explained, prim_ids
from instancing_common import flat_ids, make_instances, world_rays


@pytest.fixture(scope="module")
def inst(rq):
    return make_instances(rq)


def _tlas_host(rq, blas, M, bi):
    bounds = np.array([list(b.info["bounds_lo"]) + list(b.info["bounds_hi"]) for b in blas], np.float32)
    return rq.build_tlas_host(bounds, M, bi)


def test_tlas_host_layout(rq, inst):
    meshes, blas, M, bi, flat, tri_off = inst
    top = _tlas_host(rq, blas, M, bi)
    rows = top.woop.reshape(-1, 3, 4)
    mp = top.prim_index.reshape(-1, 3)
    assert rows.shape[0] == M.shape[0] and sorted(mp[:, 0]) == list(range(M.shape[0]))
    assert (mp[:, 1] == bi[mp[:, 0]]).all() and (mp[:, 2] == -1).all()
    for k, r in zip(mp[:, 0], rows):  # rows = world-to-object = inverse of the instance transform
        A = np.eye(4)
        A[:3, :] = M[k]
        Ainv = np.linalg.inv(A)[:3]
        assert np.allclose(r, Ainv, rtol=1e-5, atol=1e-5)


def test_tlas_host_rejects_bad_input(rq, inst):
    meshes, blas, M, bi, flat, tri_off = inst
    bounds = np.zeros((len(blas), 6), np.float32)
    bad = M.copy()
    bad[3, :, :3] = 0  # singular
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.build_tlas_host(bounds, bad, bi)
    bad = M.copy()
    bad[2, 0, 3] = np.nan
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.build_tlas_host(bounds, bad, bi)
    b2 = bi.copy()
    b2[0] = len(blas)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.build_tlas_host(bounds, M, b2)


def test_single_instance_root_leaf(rq, po, inst):
    """One identity instance equals the bottom-level scene itself."""
    meshes, blas, M, bi, flat, tri_off = inst
    hb = blas[0]
    top = _tlas_host(rq, blas[:1], np.eye(3, 4, dtype=np.float32)[None], np.zeros(1, np.int32))
    V, I = meshes[0]
    rays = world_rays(5000, 3)
    rays[:, 0:3] = np.random.default_rng(3).uniform(V.min(0), V.max(0), (5000, 3))
    for anyh in (False, True):
        got, gi = po.trace_instanced({"nodes": top.nodes, "rows": top.woop, "map": top.prim_index},
                                     [(hb.nodes, hb.woop)], rays, anyh)
        want = po.trace(0, hb.nodes, hb.woop, rays, anyh)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert ((gi == 0) == (want[:, 1].view(np.int32) >= 0)).all()


@pytest.mark.parametrize("any_hit", [False, True], ids=["closest", "any"])
def test_oracle_instanced_equals_flattened(rq, po, inst, any_hit):
    meshes, blas, M, bi, flat, tri_off = inst
    top = _tlas_host(rq, blas, M, bi)
    rays = world_rays(20000, 7)
    got, gi = po.trace_instanced({"nodes": top.nodes, "rows": top.woop, "map": top.prim_index},
                                 [(b.nodes, b.woop) for b in blas], rays, any_hit)
    FV, FI = flat
    fb = rq.HostBVH(FV, FI, rq.CWBVH)
    want = po.trace(0, fb.nodes, fb.woop, rays, any_hit)
    g = flat_ids(got, gi, blas, bi, tri_off)
    w = prim_ids(want, fb.prim_index)
    assert ((g >= 0) == (gi >= 0)).all()
    bad = np.nonzero((g >= 0) != (w >= 0))[0] if any_hit else np.nonzero(g != w)[0]
    unexplained = [i for i in bad if not _explained(po, rays[i], FV, FI, (int(g[i]), int(w[i])))]
    assert not unexplained, (len(bad), unexplained[:10])
    assert (w >= 0).sum() > 1000
    if not any_hit:
        same = (g == w) & (g >= 0)
        for i in np.nonzero(same)[0]:
            v0, v1, v2 = FV[FI[g[i]]].astype(np.float64)
            n = np.cross(v1 - v0, v2 - v0)
            cos = abs(n @ rays[i, 4:7]) / np.linalg.norm(n)
            t64 = po.tri_f64(rays[i], v0, v1, v2)[0]
            assert abs(got[i, 0] - t64) <= 1e-4 * abs(t64) + 1e-6 / max(cos, 0.01), (i, got[i, 0], t64, cos)
