"""AO ray generation and surfel sampling on the GPU against the oracle's
restatement (same Philox stream; host sinf/cosf differ by ulps, hence the
tolerance), the reference-shaped GenerateAORaysUniform, and the reference's
own generator (curand) in distribution."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_aorays_match_oracle(rq, po):
    import torch
    rng = np.random.default_rng(0)
    n, spp = 5000, 8
    pos = np.concatenate([rng.uniform(-5, 5, (n, 3)), np.ones((n, 1))], 1).astype(np.float32)
    nr = rng.normal(size=(n, 3))
    nr /= np.linalg.norm(nr, axis=1, keepdims=True)
    nr[:10] = [0, 0, 1]  # n x z == 0: the n x y fallback
    nrm = np.concatenate([nr, np.zeros((n, 1))], 1).astype(np.float32)
    rad = rng.uniform(0, 0.1, n).astype(np.float32)
    got = rq.aorays(torch.from_numpy(pos).cuda(), torch.from_numpy(nrm).cuda(), torch.from_numpy(rad).cuda(), spp,
                    seed=42, tmin=0.001, tmax=3.0, offset_scale=0.5).cpu().numpy()
    want = po.aorays(pos, nrm, rad, spp, 42, 0.001, 3.0, 0.5)
    assert np.abs(got[:, 0:3] - want[:, 0:3]).max() < 1e-5
    assert np.abs(got[:, 4:7] - want[:, 4:7]).max() < 2e-5
    assert (got[:, 3] == np.float32(0.001)).all() and (got[:, 7] == np.float32(3.0)).all()
    c = np.einsum("ij,ij->i", got[:, 4:7], np.repeat(nr, spp, axis=0))
    assert abs(c.mean() - 2 / 3) < 5e-3 and (c > -1e-5).all()


def test_surfels_on_triangles(rq):
    import torch
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    v, i = torch.from_numpy(V).cuda(), torch.from_numpy(I).cuda()
    pos, nrm, rad = rq.sample_surfels(v, i, 20000, seed=3)
    pos2, _, _ = rq.sample_surfels(v, i, 20000, seed=3)
    assert torch.equal(pos, pos2)
    p = pos.cpu().numpy()[:, :3]
    nn = nrm.cpu().numpy()[:, :3]
    assert np.allclose(np.linalg.norm(nn, axis=1), 1, atol=1e-5)
    assert (rad.cpu().numpy() == 0).all()
    assert (p >= V.min(0) - 1e-6).all() and (p <= V.max(0) + 1e-6).all()


def test_generate_ao_rays_uniform_dropin(rq):
    """Reference semantics: tmin 0.01, tmax 1e20, origin + n * r / 2, rays of
    a texel contiguous (src/ValidationKernels.cu:79-100)."""
    n, spp = 300, 32
    pos = np.zeros((n, 4), np.float32)
    pos[:, 0] = np.arange(n)
    nrm = np.tile(np.array([[0, 0, 1, 0]], np.float32), (n, 1))
    rad = np.full(n, 0.2, np.float32)
    rays = rq.GenerateAORaysUniform(n, spp, pos, nrm, rad).cpu().numpy()
    assert rays.shape == (n * spp, 8)
    assert np.allclose(rays[:, 0], np.repeat(np.arange(n), spp))
    assert np.allclose(rays[:, 2], 0.1)
    assert (rays[:, 3] == np.float32(0.01)).all() and (rays[:, 7] == np.float32(1e20)).all()
    assert abs(rays[:, 6].mean() - 2 / 3) < 1e-2


def test_reference_generator_same_distribution(rq, po):
    """The reference's curand-based generator (oracle/_ref) and this one give
    the same cosine lobe and origin offsets."""
    import ctypes as C
    import torch
    if not po.ref_available():
        pytest.skip("oracle/_ref not built")
    lib = po.ref()
    n, spp = 2000, 32
    pos = np.zeros((n, 4), np.float32)
    nrm = np.tile(np.array([[0, 0.6, 0.8, 0]], np.float32), (n, 1))
    rad = np.full(n, 0.5, np.float32)
    p = lib.ref_aorays(n, spp, pos.ctypes.data, nrm.ctypes.data, rad.ctypes.data)
    assert p
    out = torch.empty((n * spp, 8), device="cuda")
    rq.check(rq.lib.rq_device_copy(out.data_ptr(), p, n * spp * 32), "copy")
    lib.ref_cuda_free(C.c_void_p(p))
    ref = out.cpu().numpy()
    mine = rq.GenerateAORaysUniform(n, spp, pos, nrm, rad).cpu().numpy()
    # The reference's sqrtf(1 - x^2 - y^2) (src/ValidationKernels.cu:60) can
    # see a tiny negative argument under -use_fast_math and return NaN; this
    # generator clamps it at 0.
    ref_finite = np.isfinite(ref[:, 4:7]).all(axis=1)
    assert ref_finite.mean() > 0.99
    assert np.isfinite(mine).all()
    for r in (ref[ref_finite], mine):
        c = r[:, 4:7] @ np.array([0, 0.6, 0.8], np.float32)
        assert abs(c.mean() - 2 / 3) < 5e-3 and abs((c ** 2).mean() - 0.5) < 5e-3
    assert np.allclose(ref[:, 0:4], mine[:, 0:4], atol=1e-6)
    assert np.array_equal(ref[:, 7], mine[:, 7])


def test_ao_reduce(rq):
    import torch
    n, spp = 1000, 16
    hits = torch.zeros((n * spp, 4), device="cuda")
    ids = torch.randint(-1, 5, (n * spp,), device="cuda", dtype=torch.int32)
    hits[:, 1] = ids.view(torch.float32)
    ao = rq.ao_reduce(hits, n, spp).cpu().numpy()
    want = (ids.cpu().numpy().reshape(n, spp) != -1).mean(axis=1)
    assert np.allclose(ao, want)


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_trace_ao_fused_equals_trace_then_reduce(rq, kind):
    """rq_trace_ao (counts in the trace epilogue, no hit buffer) equals
    any-hit rq_trace followed by rq_ao_reduce, surfel by surfel."""
    import torch
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(2)
    ds = W.upload(V, I, kind)
    spp = 8
    rays = W.ao_rays(ds, 40_000 * spp, seed=21, spp=spp)
    ctx = rq.Context()
    hits = torch.empty((rays.shape[0], 4), device="cuda")
    rq.trace(ctx, ds.scene, rays, hits, rq.ANY)
    want = rq.ao_reduce(hits, rays.shape[0] // spp, spp)
    counts = rq.trace_ao(ctx, ds.scene, rays, spp)
    ctx.check()
    assert torch.equal(counts.float() / spp, want)
    assert 0 < int(counts.sum()) < rays.shape[0]
    rq.trace_ao(ctx, ds.scene, rays, spp, occluded=counts)  # accumulates
    assert torch.equal(counts.float() / (2 * spp), want)
    with pytest.raises(ValueError):
        rq.trace_ao(ctx, ds.scene, rays[:-1], spp)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.check(rq.lib.rq_trace_ao(ctx._h, ds.scene._h, rays.data_ptr(), rays.shape[0] - 1, spp,
                                    counts.data_ptr(), None, None), "rq_trace_ao")
