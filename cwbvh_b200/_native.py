"""ctypes bindings of librq.so (declarations in include/rq.h).

The library is loaded from this package directory only; importing fails
loudly if it has not been built (``python -m cwbvh_b200.build``), so no code
path can silently fall back to anything else.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import os

# RQ_LIBRARY points at another build of librq.so (for comparing builds);
# by default the in-tree library next to this file is loaded.
LIB_PATH = Path(os.environ.get("RQ_LIBRARY") or (Path(__file__).resolve().parent / "librq.so"))

if not LIB_PATH.exists():
    raise ImportError(f"{LIB_PATH} is missing: build it with `python cwbvh_b200/build.py`")

lib = C.CDLL(str(LIB_PATH))

i32, i64, u64, f32 = C.c_int32, C.c_int64, C.c_uint64, C.c_float
vp, cp = C.c_void_p, C.c_char_p
P = C.POINTER

RQ_OK = 0
STATUS = {
    0: "RQ_OK", 1: "RQ_ERR_INVALID_ARG", 2: "RQ_ERR_OOM", 3: "RQ_ERR_STACK_OVERFLOW", 4: "RQ_ERR_TIMEOUT",
    5: "RQ_ERR_CUDA", 6: "RQ_ERR_BAD_SCENE", 7: "RQ_ERR_NOT_FOUND", 8: "RQ_ERR_BUDGET", 9: "RQ_ERR_CANCELLED",
    10: "RQ_ERR_NO_DEVICE",
}
CWBVH, BVH2 = 0, 1
CLOSEST, ANY = 0, 1


class RQError(RuntimeError):
    def __init__(self, status: int, where: str):
        self.status = status
        detail = lib.rq_last_error().decode() if status == 5 else ""
        super().__init__(f"{where}: {STATUS.get(status, status)} {detail}".strip())


class Launch(C.Structure):
    _fields_ = [("block_size", C.c_int), ("blocks_per_sm", C.c_int), ("smem_stack", C.c_int),
                ("postpone_ratio", f32), ("fetch_nd", C.c_int), ("fetch_nw", C.c_int), ("step_limit", C.c_int)]


class BuildParams(C.Structure):
    _fields_ = [("max_leaf_size", C.c_int), ("sah_bins", C.c_int), ("max_depth", C.c_int), ("threads", C.c_int),
                ("presplit", C.c_int), ("treelet_passes", C.c_int), ("spatial_splits", C.c_int)]


class BVHInfo(C.Structure):
    _fields_ = [("node_float4s", i64), ("woop_float4s", i64), ("prim_index_count", i64), ("node_count", i64),
                ("leaf_count", i64), ("depth", i32), ("kind", i32), ("bounds_lo", f32 * 3), ("bounds_hi", f32 * 3)]


class BatchItem(C.Structure):
    _fields_ = [("scene", vp), ("rays", vp), ("hits", vp), ("count", i64)]


class BatchParams(C.Structure):
    _fields_ = [("launch", Launch), ("sort_threshold", i64), ("use_graph", C.c_int)]


class ServerParams(C.Structure):
    _fields_ = [("hbm_budget_bytes", i64), ("max_batch_rays", i64), ("streams", C.c_int), ("query", C.c_int),
                ("launch", Launch)]


class RequestStats(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("start_ms", C.c_double), ("done_ms", C.c_double), ("rays", i64),
                ("batch_id", i32), ("status", i32)]


class ServerMemoryStats(C.Structure):
    _fields_ = [("pool_bytes", i64), ("in_use_bytes", i64), ("peak_in_use_bytes", i64), ("admission_waits", i64),
                ("pieces", i64), ("max_batch_rays", i64)]


def _sig(name, res, *args):
    fn = getattr(lib, name)
    fn.restype = res
    fn.argtypes = list(args)
    return fn


_sig("rq_status_string", cp, C.c_int)
_sig("rq_last_error", cp)
_sig("rq_version", cp)
_sig("rq_device_sm_count", C.c_int)
_sig("rq_build_bvh", C.c_int, vp, i64, vp, i64, C.c_int, P(BuildParams), P(vp))
_sig("rq_host_bvh_info", C.c_int, vp, P(BVHInfo))
_sig("rq_host_bvh_buffers", C.c_int, vp, P(vp), P(vp), P(vp))
_sig("rq_host_bvh_free", None, vp)
_sig("rq_host_bvh_tree", C.c_int, vp, P(i32), P(i64), P(i64), P(i64), P(i32), vp, vp, vp, vp, vp)
_sig("rq_woopify", C.c_int, vp, vp, vp, vp)
_sig("rq_scene_create", C.c_int, C.c_int, vp, i64, vp, i64, vp, i64, C.c_int, P(vp))
_sig("rq_scene_from_host_bvh", C.c_int, vp, P(vp))
_sig("rq_scene_destroy", C.c_int, vp)
_sig("rq_scene_device_buffers", C.c_int, vp, P(vp), P(vp), P(vp))
_sig("rq_scene_bytes", i64, vp)
_sig("rq_ctx_create", C.c_int, P(vp))
_sig("rq_ctx_destroy", C.c_int, vp)
_sig("rq_ctx_check", C.c_int, vp, vp)
_sig("rq_trace", C.c_int, vp, vp, vp, vp, i64, C.c_int, P(Launch), vp)
_sig("rq_trace_counted", C.c_int, vp, vp, vp, vp, i64, C.c_int, vp, vp, vp)
_sig("rq_trace_ordered", C.c_int, vp, vp, vp, vp, i64, C.c_int, vp)
_sig("rq_default_launch", C.c_int, C.c_int, C.c_int, P(Launch))
_sig("rq_aorays", C.c_int, vp, vp, vp, i64, C.c_int, u64, f32, f32, f32, vp, vp)
_sig("rq_sample_surfels", C.c_int, vp, vp, i64, i64, u64, vp, vp, vp, vp)
_sig("rq_ao_reduce", C.c_int, vp, i64, C.c_int, vp, vp)
_sig("rq_sort_rays", C.c_int, vp, vp, i64, vp, vp, vp, vp, vp)
_sig("rq_batch_create", C.c_int, vp, P(BatchItem), C.c_int, C.c_int, P(BatchParams), P(vp))
_sig("rq_batch_run", C.c_int, vp, vp)
_sig("rq_batch_destroy", C.c_int, vp)
_sig("rq_batch_run_stage", C.c_int, vp, C.c_int, vp)
_sig("rq_batch_kernel_count", C.c_int, vp)
_sig("rq_batch_total_rays", i64, vp)
_sig("rq_autotune", C.c_int, vp, vp, vp, vp, i64, C.c_int, cp, P(Launch), vp)
_sig("rq_autotune_batch", C.c_int, vp, P(BatchItem), C.c_int, C.c_int, cp, P(BatchParams), vp)
_sig("rq_server_create", C.c_int, P(ServerParams), P(vp))
_sig("rq_server_add_scene", C.c_int, vp, vp, P(i32))
_sig("rq_server_submit", C.c_int, vp, i32, vp, vp, i64, P(u64))
_sig("rq_server_wait", C.c_int, vp, u64, i64, P(RequestStats))
_sig("rq_server_cancel", C.c_int, vp, u64)
_sig("rq_server_destroy", C.c_int, vp)
_sig("rq_server_memory", C.c_int, vp, P(ServerMemoryStats))
_sig("rq_gen_heightfield_boxes", C.c_int, u64, C.c_int, C.c_int, f32, f32, P(vp), P(i64), P(vp), P(i64))
_sig("rq_gen_city", C.c_int, u64, C.c_int, P(vp), P(i64), P(vp), P(i64))
_sig("rq_gen_spheres_terrain", C.c_int, u64, i64, P(vp), P(i64), P(vp), P(i64))
_sig("rq_free_mesh", None, vp, vp)
_sig("rq_rtBindCWBVHData", C.c_int, vp, vp, vp)
_sig("rq_rtTraceCWBVH", C.c_int, vp, vp, C.c_int)
_sig("rq_rtBindBVH2Data", C.c_int, vp, vp, vp)
_sig("rq_rtTraceBVH2", C.c_int, vp, vp, C.c_int)
_sig("rq_rtOccludedCWBVH", C.c_int, vp, vp, C.c_int)
_sig("rq_rtOccludedBVH2", C.c_int, vp, vp, C.c_int)
_sig("rq_GenerateAORaysUniform", vp, C.c_int, C.c_int, vp, vp, vp)
_sig("rq_device_copy", C.c_int, vp, vp, i64)
_sig("rq_device_free", C.c_int, vp)

# scene files, GPU build, sizes
_sig("rq_convert_tree", C.c_int, i32, i64, vp, vp, i64, vp, vp, i64, vp, i32, vp, i64, vp, i64, P(vp))
_sig("rq_load_mesh_dat", C.c_int, cp, P(vp), P(i64), P(vp), P(i64), P(vp))
_sig("rq_save_mesh_dat", C.c_int, cp, vp, i64, vp, i64, vp)
_sig("rq_load_samplecache_dat", C.c_int, cp, P(i32), P(i32), P(vp), P(vp), P(vp))
_sig("rq_save_samplecache_dat", C.c_int, cp, i32, i32, vp, vp, vp)
_sig("rq_free_host", None, vp)
_sig("rq_host_bvh_save", C.c_int, vp, cp)
_sig("rq_host_bvh_load", C.c_int, cp, P(vp))
_sig("rq_build_scene_gpu", C.c_int, vp, i64, vp, i64, C.c_int, C.c_int, C.c_int, P(vp), vp)
_sig("rq_scene_sizes", C.c_int, vp, P(i64), P(i64), P(i64))
# rays and AO
_sig("rq_sort_rays_static", C.c_int, vp, i64, vp, vp, vp, vp, vp)
_sig("rq_camera_rays", C.c_int, vp, vp, vp, f32, C.c_int, C.c_int, f32, f32, vp, vp)
_sig("rq_camera_rays_tiled", C.c_int, vp, vp, vp, f32, C.c_int, C.c_int, C.c_int, C.c_int, f32, f32, vp, vp)
_sig("rq_surfels_from_hits", C.c_int, vp, vp, vp, i64, vp, vp, vp, vp)
_sig("rq_probe_l2_read", C.c_int, vp, i64, C.c_int, vp, vp)
_sig("rq_probe_l2_read_shape", C.c_int, vp, i64, C.c_int, C.c_int, C.c_int, vp, vp)
_sig("rq_trace_ao", C.c_int, vp, vp, vp, i64, C.c_int, vp, P(Launch), vp)
# instancing
_sig("rq_tlas_create", C.c_int, P(vp), C.c_int, vp, vp, i64, P(vp))
_sig("rq_tlas_destroy", C.c_int, vp)
_sig("rq_tlas_buffers", C.c_int, vp, P(vp), P(i64), P(vp), P(i64), P(vp))
_sig("rq_trace_instanced", C.c_int, vp, vp, vp, vp, vp, i64, C.c_int, P(Launch), vp)
_sig("rq_tlas_build_host", C.c_int, vp, C.c_int, vp, vp, i64, P(vp))
# one ray set over several devices
_sig("rq_shard_range", C.c_int, i64, C.c_int, C.c_int, P(i64), P(i64))
_sig("rq_sharded_create", C.c_int, C.c_int, vp, vp, i64, P(vp))
_sig("rq_sharded_trace", C.c_int, vp, vp, vp, i64, C.c_int, P(Launch), vp)
_sig("rq_sharded_destroy", C.c_int, vp)
# serving
_sig("rq_server_submit_bake", C.c_int, vp, i32, vp, vp, vp, i64, C.c_int, u64, f32, f32, f32, vp, P(u64))


def check(status: int, where: str) -> None:
    if status != RQ_OK:
        raise RQError(status, where)
