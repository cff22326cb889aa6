"""rq_sort_rays_static -- the Morton ray sort for callers that cannot call
cudaMalloc (a plugin whose host owns all device memory through its own pool,
a service whose device-memory budget was fixed at start-up).  It keeps its
scratch in a static device array instead of allocating.  Through the C ABI,
two calls in a row must give the same sorted rays and permutation as
rq_sort_rays, the allocating entry point; once the first calls have run,
further calls must leave the device's free memory unchanged; and a count
above the array's limit must be refused with a clear error.

This file is collected last so that a failure here stops a run only after
every other test has run."""
import ctypes as C

import pytest

pytestmark = pytest.mark.gpu

MAX_RAYS = 524288  # RQ_SORT_STATIC_MAX_RAYS in include/rq.h


def _static_sort(rq, rays, lo, hi, out=None, perm=None):
    import torch
    n = rays.shape[0]
    if out is None:
        out = torch.empty_like(rays)
        perm = torch.full((n,), -1, dtype=torch.int32, device=rays.device)
    st = rq.lib.rq_sort_rays_static(rays.data_ptr(), n, (C.c_float * 3)(*lo), (C.c_float * 3)(*hi),
                                    out.data_ptr(), perm.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == 0, rq.lib.rq_last_error()
    torch.cuda.synchronize()
    return out, perm


def _scene(rq):
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    ds = W.upload(V, I, rq.CWBVH)
    return ds, ds.host.info["bounds_lo"], ds.host.info["bounds_hi"]


def test_static_sort_matches_allocating_sort_twice(rq):
    import torch
    from cwbvh_b200 import workloads as W
    ds, lo, hi = _scene(rq)
    ctx = rq.Context()
    # Two calls in a row on different ray sets: the second must not see the
    # first one's leftovers in the shared scratch.
    for n, seed in ((MAX_RAYS, 1000), (123_457, 2000)):
        rays = W.ao_rays(ds, n, seed=seed)
        got_rays, got_perm = _static_sort(rq, rays, lo, hi)
        want_rays, want_perm = rq.sort_rays(ctx, rays, lo, hi)
        torch.cuda.synchronize()
        assert torch.equal(got_perm, want_perm)
        assert torch.equal(got_rays, want_rays)
        assert torch.equal(got_rays, rays[got_perm.long()])


def test_static_sort_allocates_nothing(rq):
    import torch
    from cwbvh_b200 import workloads as W
    ds, lo, hi = _scene(rq)
    cases = []
    for n, seed in ((MAX_RAYS, 3000), (77_777, 4000)):
        rays = W.ao_rays(ds, n, seed=seed)
        cases.append((rays, torch.empty_like(rays), torch.empty((n,), dtype=torch.int32, device="cuda")))
    # The first calls set up the device and load the kernels they launch.
    for rays, out, perm in cases:
        _static_sort(rq, rays, lo, hi, out, perm)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for rays, out, perm in cases:
            _static_sort(rq, rays, lo, hi, out, perm)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    rays, out, perm = cases[1]
    assert torch.equal(out, rays[perm.long()])


def test_static_sort_refuses_more_than_its_limit(rq):
    import torch
    lo = (C.c_float * 3)(0, 0, 0)
    hi = (C.c_float * 3)(1, 1, 1)
    dummy = torch.empty(8, device="cuda")
    st = rq.lib.rq_sort_rays_static(dummy.data_ptr(), MAX_RAYS + 1, lo, hi, dummy.data_ptr(), dummy.data_ptr(),
                                    None)
    assert st == 1  # RQ_ERR_INVALID_ARG
    msg = rq.lib.rq_last_error().decode()
    assert str(MAX_RAYS) in msg and "rq_sort_rays" in msg
    assert rq.lib.rq_sort_rays_static(dummy.data_ptr(), 0, lo, hi, dummy.data_ptr(), dummy.data_ptr(), None) == 0
