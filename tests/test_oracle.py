"""The CPU oracle pinned against known answers and the reference's own output.

* the reference's validation scene (src/ValidationKernels.cu:6-39), whose
  closest hits follow analytically;
* the reference kernels' recorded results (tests/golden/trace_fixtures.npz,
  made on a B200 by tests/golden/make_golden.py --traces) -- equal up to
  FP64-adjudicated ties, the reference computing 1/x approximately;
* Philox4x32-10 known-answer vectors (Salmon et al., SC 2011);
* layout independence: CWBVH and BVH2 give the same answers on the same rays.
"""
from pathlib import Path

import numpy as np
import pytest

from adjudicate import compare, prim_ids

GOLD = Path(__file__).resolve().parent / "golden"


def quads(n=1000, r=5000):
    tid = np.arange(n)
    V = np.zeros((3 * n, 3), np.float32)
    V[0::3] = np.stack([np.full(n, -1.1), np.full(n, -1.1), tid], 1)
    V[1::3] = np.stack([np.full(n, 1.1), np.full(n, -1.1), tid], 1)
    V[2::3] = np.stack([np.full(n, 1.1), np.full(n, 1.1), tid], 1)
    I = np.arange(3 * n, dtype=np.int32).reshape(-1, 3)
    rid = np.arange(r, dtype=np.int64)
    # rayId * 12345678 % Count in 32-bit signed arithmetic, C remainder
    k = np.fmod(((rid * 12345678) & 0xFFFFFFFF).astype(np.uint32).view(np.int32).astype(np.int64), n)
    d = np.array([-0.01, 0.5, 1.0])
    d = d / np.linalg.norm(d)
    rays = np.zeros((r, 8), np.float32)
    rays[:, 0], rays[:, 1], rays[:, 2], rays[:, 3] = 0.5, -0.5, k - 0.5, 0.0
    rays[:, 4:7] = d
    rays[:, 7] = 1e20
    # The ray crosses plane m at offset (m - z0) (-0.01, 0.5) / 1; it is
    # inside the triangle for m - z0 < ~1.96: plane k from z0 = k - 0.5, or
    # plane 0 from z0 = -1.5; farther below it misses every plane.
    expect = np.where(k >= 0, k, np.where(k == -1, 0, -1))
    return V, I, rays, expect


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_known_answer_quads(rq, po, kind):
    V, I, rays, expect = quads()
    hb = rq.HostBVH(V, I, kind)
    h = po.trace(kind, hb.nodes, hb.woop, rays, False)
    assert np.array_equal(prim_ids(h, hb.prim_index), expect)
    hit = expect >= 0
    t_exact = (expect[hit] - rays[hit, 2].astype(np.float64)) / rays[hit, 6]
    assert np.allclose(h[hit, 0], t_exact, rtol=0, atol=1e-4)  # z0 ~ 1e3 carries 6e-5 of float spacing
    assert (h[~hit, 0] == np.float32(1e20)).all()
    ha = po.trace(kind, hb.nodes, hb.woop, rays, True)
    assert np.array_equal(prim_ids(ha, hb.prim_index) >= 0, hit)


def test_layouts_agree(rq, po):
    """CWBVH and BVH2 traversal of the same rays give the same answers."""
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    rng = np.random.default_rng(2)
    n = 40_000
    tri = rng.integers(0, I.shape[0], n)
    a, b = np.sqrt(rng.random(n)), rng.random(n)
    P = V[I[tri, 0]] * (1 - a)[:, None] + V[I[tri, 1]] * (b * a)[:, None] + V[I[tri, 2]] * (a - b * a)[:, None]
    Nn = np.cross(V[I[tri, 1]] - V[I[tri, 0]], V[I[tri, 2]] - V[I[tri, 0]])
    Nn /= np.linalg.norm(Nn, axis=1, keepdims=True)
    pos = np.concatenate([P, np.ones((n, 1))], 1).astype(np.float32)
    nrm = np.concatenate([Nn, np.zeros((n, 1))], 1).astype(np.float32)
    dg = float(np.linalg.norm(V.max(0) - V.min(0)))
    rays = po.aorays(pos, nrm, None, 1, 7, 1e-4 * dg, 0.1 * dg, 0.0)
    cw = rq.HostBVH(V, I, rq.CWBVH)
    b2 = rq.HostBVH(V, I, rq.BVH2)
    for any_hit in (False, True):
        h1 = po.trace(0, cw.nodes, cw.woop, rays, any_hit)
        h2 = po.trace(1, b2.nodes, b2.woop, rays, any_hit)
        i1, i2 = prim_ids(h1, cw.prim_index), prim_ids(h2, b2.prim_index)
        if any_hit:
            assert np.array_equal(i1 >= 0, i2 >= 0)
        else:
            assert np.array_equal(i1, i2)
            assert np.array_equal(h1[:, 0], h2[:, 0])  # same Woop rows, same t


def test_philox_known_answers(po):
    kat = [((0, 0, 0, 0), 0, (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
           ((0xFFFFFFFF,) * 4, 0xFFFFFFFFFFFFFFFF, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
           ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), 0xA4093822 | (0x299F31D0 << 32),
            (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]
    for ctr, key, want in kat:
        assert po.philox(np.array(ctr, np.uint32), key).tolist() == list(want)


def test_aorays_cosine_lobe(po):
    """Directions are cosine-distributed about the normal: E[cos] = 2/3,
    E[cos^2] = 1/2 (src/ValidationKernels.cu:41-61 semantics)."""
    n = 200_000
    pos = np.zeros((1, 4), np.float32)
    for nrm in ([0, 0, 1, 0], [0.6, 0, 0.8, 0], [0, 1, 0, 0]):
        r = po.aorays(pos, np.array([nrm], np.float32), np.array([2.0], np.float32), n, 11, 0.01, 1e20, 0.5)
        c = r[:, 4:7] @ np.array(nrm[:3], np.float32)
        assert abs(c.mean() - 2 / 3) < 5e-3 and abs((c ** 2).mean() - 0.5) < 5e-3
        assert (c >= -1e-6).all()
        assert np.allclose(np.linalg.norm(r[:, 4:7], axis=1), 1, atol=1e-5)
        assert np.allclose(r[:, 0:3], 0.5 * 2.0 * np.array(nrm[:3]), atol=1e-6)  # origin offset radius/2
        assert (r[:, 3] == np.float32(0.01)).all() and (r[:, 7] == np.float32(1e20)).all()


def test_aorays_zero_normal_is_empty_ray(po):
    """A surfel without a surface (a primary miss) yields empty rays:
    origin at the surfel, tmin = tmax = 0, so no traversal can report a hit."""
    pos = np.array([[1, 2, 3, 1], [4, 5, 6, 1]], np.float32)
    nrm = np.array([[0, 0, 0, 0], [0, 0, 1, 0]], np.float32)
    r = po.aorays(pos, nrm, np.array([0.5, 0.5], np.float32), 3, 5, 0.01, 9.0, 1.0)
    assert np.array_equal(r[:3], np.tile(np.array([1, 2, 3, 0, 0, 0, 1, 0], np.float32), (3, 1)))
    assert (r[3:, 3] == np.float32(0.01)).all() and (r[3:, 7] == np.float32(9.0)).all()


def test_adjudicator_f64(po):
    ray = np.array([0.25, 0.25, -1, 0, 0, 0, 1, 10], np.float32)
    t, u, v, det = po.tri_f64(ray, [1, 0, 0], [0, 1, 0], [0, 0, 0])
    assert abs(t - 1) < 1e-12 and abs(u - 0.25) < 1e-12 and abs(v - 0.25) < 1e-12


@pytest.mark.skipif(not (GOLD / "trace_fixtures.npz").exists(), reason="needs tests/golden/trace_fixtures.npz")
@pytest.mark.parametrize("tag,kind", [("cw", 0), ("b2", 1)])
def test_oracle_matches_reference_kernels(rq, po, tag, kind):
    """The oracle against rtTraceCWBVH / rtTraceBVH2 run on a B200."""
    fx = np.load(GOLD / "trace_fixtures.npz")
    V, I, rays = fx["V"], fx["I"], fx["rays"]
    ref = fx[f"{tag}/ref_hits"]
    # The reference's persistent CWBVH loop drops a few rays (never written,
    # still the NaN pre-fill); they are excluded.
    written = ~np.isnan(ref[:, 0])
    assert written.mean() > 0.98
    rays, ref = rays[written], ref[written]
    want = po.trace(kind, fx[f"{tag}/nodes"], fx[f"{tag}/woop"], rays, False)
    res = compare(po, rays, ref, want, fx[f"{tag}/prim"], V, I, any_hit=False)
    assert res["hits"] > rays.shape[0] // 10
    # any-hit occlusion bits follow from the closest-hit ids
    wa = po.trace(kind, fx[f"{tag}/nodes"], fx[f"{tag}/woop"], rays, True)
    compare(po, rays, ref, wa, fx[f"{tag}/prim"], V, I, any_hit=True)
