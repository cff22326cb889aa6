"""cwbvh_b200 -- a B200 ray-query engine for compressed wide BVHs.

Python front end over librq.so (C ABI in include/rq.h).  Host BVH build and
conversion run in C++; tracing, ray generation, sorting, batching and serving
run in hand-written sm_100a CUDA kernels.  Device buffers are torch CUDA
tensors (torch is used for device memory and streams only).

Reference entry points mirrored here (names and argument meaning):
  rtBindCWBVHData / rtTraceCWBVH   src/TraversalKernelCWBVH.h:3-11
  rtBindBVH2Data  / rtTraceBVH2    src/TraversalKernelBVH2.h:3-11
  GenerateAORaysUniform            src/ValidationKernels.h:3-9
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, Optional, Sequence

import numpy as np

from . import _native as N
from ._native import ANY, BVH2, CLOSEST, CWBVH, Launch, RQError, check, lib

GPU_BUILD_LBVH = 0  # rq_build_scene_gpu: Karras radix tree over the Morton order
GPU_BUILD_PLOC = 1  # rq_build_scene_gpu: parallel locally-ordered clustering
GPU_BUILD_THREAD_TREELETS = 0x100  # OR-ed into the method: one thread per treelet (same trees, slower)

__all__ = [
    "ANY", "BVH2", "CLOSEST", "CWBVH", "GPU_BUILD_LBVH", "GPU_BUILD_PLOC", "Launch", "RQError", "HostBVH", "Scene", "Context", "Batch", "Server",
    "trace", "trace_ordered", "trace_counted", "aorays", "sample_surfels", "ao_reduce", "sort_rays",
    "autotune", "autotune_batch", "default_launch", "woopify", "gen_heightfield_boxes", "gen_city",
    "gen_spheres_terrain", "rtBindCWBVHData", "rtTraceCWBVH", "rtBindBVH2Data", "rtTraceBVH2",
    "rtOccludedCWBVH", "rtOccludedBVH2", "GenerateAORaysUniform", "version", "lib", "camera_rays",
    "surfels_from_hits", "trace_ao", "Tlas", "trace_instanced", "build_tlas_host", "load_mesh_dat", "save_mesh_dat", "load_samplecache_dat", "save_samplecache_dat",
]


def version() -> str:
    return lib.rq_version().decode()


# ------------------------------------------------------------ helpers ----

def _ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (must be contiguous)."""
    if t is None:
        return 0
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class _On:
    """Allocate on the stream the work goes to (no-op for the current stream)."""

    def __init__(self, stream):
        self.stream = stream
        self.ctx = None

    def __enter__(self):
        if self.stream is not None and not isinstance(self.stream, int):
            import torch
            self.ctx = torch.cuda.stream(self.stream)
            self.ctx.__enter__()

    def __exit__(self, *exc):
        if self.ctx is not None:
            self.ctx.__exit__(*exc)


def _rows(t, width: int, what: str) -> int:
    n = t.numel() * t.element_size()
    if n % (width * 4):
        raise ValueError(f"{what}: byte size {n} is not a multiple of {width * 4}")
    return n // (width * 4)


# ------------------------------------------------------------- meshes ----

def _take_mesh(v, nv, i, nt):
    verts = np.ctypeslib.as_array(C.cast(v, C.POINTER(C.c_float)), shape=(nv.value * 3,)).copy().reshape(-1, 3)
    idx = np.ctypeslib.as_array(C.cast(i, C.POINTER(C.c_int32)), shape=(nt.value * 3,)).copy().reshape(-1, 3)
    lib.rq_free_mesh(v, i)
    return verts, idx


def gen_heightfield_boxes(seed: int = 0, grid: int = 64, n_boxes: int = 200, box_min: float = 0.01,
                          box_max: float = 0.1):
    """(grid+1)^2-vertex heightfield over [0,1]^2 (heights U[0,1]) plus boxes."""
    v, i, nv, nt = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    check(lib.rq_gen_heightfield_boxes(seed, grid, n_boxes, box_min, box_max, C.byref(v), C.byref(nv), C.byref(i),
                                       C.byref(nt)), "rq_gen_heightfield_boxes")
    return _take_mesh(v, nv, i, nt)


def gen_city(seed: int = 0, n_buildings: int = 10000):
    v, i, nv, nt = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    check(lib.rq_gen_city(seed, n_buildings, C.byref(v), C.byref(nv), C.byref(i), C.byref(nt)), "rq_gen_city")
    return _take_mesh(v, nv, i, nt)


def gen_spheres_terrain(seed: int = 0, target_tris: int = 1_000_000):
    v, i, nv, nt = C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    check(lib.rq_gen_spheres_terrain(seed, target_tris, C.byref(v), C.byref(nv), C.byref(i), C.byref(nt)),
          "rq_gen_spheres_terrain")
    return _take_mesh(v, nv, i, nt)


def load_mesh_dat(path):
    """(vertices (nV, 3) float32, indices (nT, 3) int32, materials (nT,) int32)
    from the reference's mesh.dat format."""
    v, i, m, nv, nt = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_int64(), C.c_int64()
    check(lib.rq_load_mesh_dat(str(path).encode(), C.byref(v), C.byref(nv), C.byref(i), C.byref(nt), C.byref(m)),
          "rq_load_mesh_dat")
    mats = np.ctypeslib.as_array(C.cast(m, C.POINTER(C.c_int32)), shape=(nt.value,)).copy() if nt.value else \
        np.zeros(0, np.int32)
    lib.rq_free_host(m)
    verts, idx = _take_mesh(v, nv, i, nt)
    return verts, idx, mats


def save_mesh_dat(path, vertices, indices, materials=None) -> None:
    v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
    i = np.ascontiguousarray(indices, np.int32).reshape(-1, 3)
    m = None if materials is None else np.ascontiguousarray(materials, np.int32).reshape(-1)
    if m is not None and m.size != i.shape[0]:
        raise ValueError("materials: one per triangle")
    check(lib.rq_save_mesh_dat(str(path).encode(), v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0],
                               None if m is None else m.ctypes.data), "rq_save_mesh_dat")


def load_samplecache_dat(path):
    """(size_x, size_y, pos (n, 4), nrm (n, 4), radius (n,)) from the
    reference's samplecache.dat format, n = size_x * size_y."""
    sx, sy, p, q, r = C.c_int32(), C.c_int32(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    check(lib.rq_load_samplecache_dat(str(path).encode(), C.byref(sx), C.byref(sy), C.byref(p), C.byref(q),
                                      C.byref(r)), "rq_load_samplecache_dat")
    n = sx.value * sy.value
    take = lambda ptr, k: (np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(k,)).copy()  # noqa: E731
                           if k else np.zeros(0, np.float32))
    out = (sx.value, sy.value, take(p, 4 * n).reshape(-1, 4), take(q, 4 * n).reshape(-1, 4), take(r, n))
    for ptr in (p, q, r):
        lib.rq_free_host(ptr)
    return out


def save_samplecache_dat(path, size_x: int, size_y: int, pos, nrm, radius) -> None:
    n = size_x * size_y
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 4)
    q = np.ascontiguousarray(nrm, np.float32).reshape(-1, 4)
    r = np.ascontiguousarray(radius, np.float32).reshape(-1)
    if p.shape[0] != n or q.shape[0] != n or r.size != n:
        raise ValueError(f"sample cache arrays must hold size_x * size_y = {n} entries")
    check(lib.rq_save_samplecache_dat(str(path).encode(), size_x, size_y, p.ctypes.data, q.ctypes.data,
                                      r.ctypes.data), "rq_save_samplecache_dat")


def woopify(v0, v1, v2) -> np.ndarray:
    """3 float4 Woop rows (V0, V1, V2) of one triangle, shape (3, 4)."""
    a = [np.ascontiguousarray(x, dtype=np.float32) for x in (v0, v1, v2)]
    out = np.zeros(12, np.float32)
    check(lib.rq_woopify(*(x.ctypes.data for x in a), out.ctypes.data), "rq_woopify")
    return out.reshape(3, 4)


# ---------------------------------------------------------- host BVHs ----

class HostBVH:
    """A converted BVH in host memory (node / Woop / primitive-index buffers)."""

    def __init__(self, vertices, indices, kind: int = CWBVH, max_leaf_size: int = 0, sah_bins: int = 0,
                 max_depth: int = 0, threads: int = 0, tree: Optional[dict] = None, presplit: int = 0,
                 treelet_passes: int = 0, spatial_splits: int = 0):
        """Build with the library's SAH builder, or -- with `tree` (the dict
        shape of HostBVH.tree()) -- convert a tree built elsewhere."""
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        i = np.ascontiguousarray(indices, dtype=np.int32).reshape(-1, 3)
        self.vertices, self.indices, self.kind = v, i, kind
        h = C.c_void_p()
        if tree is None:
            bp = N.BuildParams(max_leaf_size, sah_bins, max_depth, threads, presplit, treelet_passes, spatial_splits)
            check(lib.rq_build_bvh(v.ctypes.data, v.shape[0], i.ctypes.data, i.shape[0], kind, C.byref(bp),
                                   C.byref(h)), "rq_build_bvh")
        else:
            codes = np.ascontiguousarray(tree["codes"], np.int32)
            boxes = np.ascontiguousarray(tree["boxes"], np.float32)
            lf = np.ascontiguousarray(tree["leaf_first"], np.int32)
            lc = np.ascontiguousarray(tree["leaf_count"], np.int32)
            refs = np.ascontiguousarray(tree["prim_refs"], np.int32)
            self.kind = kind = CWBVH if tree["width"] == 8 else BVH2
            check(lib.rq_convert_tree(tree["width"], codes.shape[0], codes.ctypes.data, boxes.ctypes.data,
                                      lf.size, lf.ctypes.data, lc.ctypes.data, refs.size, refs.ctypes.data,
                                      int(tree["root_is_leaf"]), v.ctypes.data, v.shape[0], i.ctypes.data,
                                      i.shape[0], C.byref(h)), "rq_convert_tree")
        self._adopt(h)

    def _adopt(self, h) -> None:
        self._h = h
        info = N.BVHInfo()
        check(lib.rq_host_bvh_info(h, C.byref(info)), "rq_host_bvh_info")
        self.info = {f: getattr(info, f) for f, _ in N.BVHInfo._fields_}
        self.info["bounds_lo"] = tuple(info.bounds_lo)
        self.info["bounds_hi"] = tuple(info.bounds_hi)
        n, w, p = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.rq_host_bvh_buffers(h, C.byref(n), C.byref(w), C.byref(p)), "rq_host_bvh_buffers")
        self.nodes = np.ctypeslib.as_array(C.cast(n, C.POINTER(C.c_float)),
                                           shape=(info.node_float4s * 4,)).copy().reshape(-1, 4)
        self.woop = (np.ctypeslib.as_array(C.cast(w, C.POINTER(C.c_float)), shape=(info.woop_float4s * 4,))
                     .copy().reshape(-1, 4) if info.woop_float4s else np.zeros((0, 4), np.float32))
        self.prim_index = (np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int32)), shape=(info.prim_index_count,))
                           .copy() if info.prim_index_count else np.zeros(0, np.int32))

    def save(self, path) -> None:
        """Write the converted buffers to a scene file (rq_host_bvh_save)."""
        check(lib.rq_host_bvh_save(self._h, str(path).encode()), "rq_host_bvh_save")

    @classmethod
    def load(cls, path) -> "HostBVH":
        """A host BVH from a scene file: buffers only, no builder tree, no mesh."""
        h = C.c_void_p()
        check(lib.rq_host_bvh_load(str(path).encode(), C.byref(h)), "rq_host_bvh_load")
        self = cls.__new__(cls)
        self.vertices = self.indices = None
        self._adopt(h)
        self.kind = self.info["kind"]
        return self

    def tree(self) -> dict:
        """The pre-conversion tree (see rq_host_bvh_tree)."""
        w, nn, nl, npr, rl = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        check(lib.rq_host_bvh_tree(self._h, C.byref(w), C.byref(nn), C.byref(nl), C.byref(npr), C.byref(rl),
                                   None, None, None, None, None), "rq_host_bvh_tree")
        W = w.value
        codes = np.zeros((nn.value, W), np.int32)
        boxes = np.zeros((nn.value, W, 6), np.float32)
        lf = np.zeros(nl.value, np.int32)
        lc = np.zeros(nl.value, np.int32)
        refs = np.zeros(npr.value, np.int32)
        check(lib.rq_host_bvh_tree(self._h, None, None, None, None, None, codes.ctypes.data, boxes.ctypes.data,
                                   lf.ctypes.data, lc.ctypes.data, refs.ctypes.data), "rq_host_bvh_tree")
        return {"width": W, "codes": codes, "boxes": boxes, "leaf_first": lf, "leaf_count": lc, "prim_refs": refs,
                "root_is_leaf": bool(rl.value)}

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_host_bvh_free(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ------------------------------------------------------- device state ----

class Scene:
    """A device-resident scene (node + Woop buffers in HBM)."""

    def __init__(self, handle: C.c_void_p, kind: int, keep=None):
        self._h = handle
        self.kind = kind
        self._keep = keep

    @classmethod
    def from_host(cls, hb: HostBVH) -> "Scene":
        h = C.c_void_p()
        check(lib.rq_scene_from_host_bvh(hb._h, C.byref(h)), "rq_scene_from_host_bvh")
        return cls(h, hb.kind)

    @classmethod
    def from_arrays(cls, kind: int, nodes: np.ndarray, woop: np.ndarray, prim_index: Optional[np.ndarray] = None):
        nodes = np.ascontiguousarray(nodes, np.float32)
        woop = np.ascontiguousarray(woop, np.float32)
        pi = None if prim_index is None else np.ascontiguousarray(prim_index, np.int32)
        h = C.c_void_p()
        check(lib.rq_scene_create(kind, nodes.ctypes.data, nodes.size // 4, woop.ctypes.data, woop.size // 4,
                                  None if pi is None else pi.ctypes.data, 0 if pi is None else pi.size, 1,
                                  C.byref(h)), "rq_scene_create")
        return cls(h, kind)

    @classmethod
    def build_gpu(cls, vertices, indices, optimize_passes: int = 2, method: int = GPU_BUILD_PLOC,
                  split_budget: int = 0, stream=None) -> "Scene":
        """CWBVH built on the device (rq_build_scene_gpu) from CUDA tensors
        vertices (nv, 3) float32 and indices (nt, 3) int32; `method` is
        GPU_BUILD_PLOC (clustering, better trees) or GPU_BUILD_LBVH (radix
        tree, fastest build); `split_budget` (percent of the triangles, 0 =
        none) lets badly fitting triangles be cut into extra references."""
        h = C.c_void_p()
        check(lib.rq_build_scene_gpu(_ptr(vertices), _rows(vertices, 3, "vertices"), _ptr(indices),
                                     _rows(indices, 3, "indices"), method, optimize_passes, split_budget,
                                     C.byref(h), _stream(stream)),
              "rq_build_scene_gpu")
        return cls(h, CWBVH)

    def download(self):
        """Host copies (nodes (n, 4) float32, woop (m, 4) float32, prim_index) of the device buffers."""
        import torch
        n, w, p = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.rq_scene_device_buffers(self._h, C.byref(n), C.byref(w), C.byref(p)), "rq_scene_device_buffers")
        nn, nw, npi = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib.rq_scene_sizes(self._h, C.byref(nn), C.byref(nw), C.byref(npi)), "rq_scene_sizes")
        out = []
        for ptr, count, width, dt in ((n, nn.value, 4, torch.float32), (w, nw.value, 4, torch.float32),
                                      (p, npi.value, 1, torch.int32)):
            t = torch.empty((count, width) if width > 1 else (count,), dtype=dt, device="cuda")
            if count:
                check(lib.rq_device_copy(t.data_ptr(), ptr, count * width * 4), "rq_device_copy")
            out.append(t.cpu().numpy())
        return tuple(out)

    @classmethod
    def from_device(cls, kind: int, nodes, woop, prim_index=None) -> "Scene":
        """Borrow device tensors (kept alive by the Scene object)."""
        h = C.c_void_p()
        check(lib.rq_scene_create(kind, _ptr(nodes), _rows(nodes, 4, "nodes"), _ptr(woop), _rows(woop, 4, "woop"),
                                  _ptr(prim_index) or None, 0 if prim_index is None else prim_index.numel(), 0,
                                  C.byref(h)), "rq_scene_create")
        return cls(h, kind, keep=(nodes, woop, prim_index))

    @property
    def nbytes(self) -> int:
        return int(lib.rq_scene_bytes(self._h))

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class Context:
    """Device scratch for the persistent kernels (ray counter, error word)."""

    def __init__(self):
        h = C.c_void_p()
        check(lib.rq_ctx_create(C.byref(h)), "rq_ctx_create")
        self._h = h

    def check(self, stream=None) -> None:
        check(lib.rq_ctx_check(self._h, _stream(stream)), "rq_ctx_check")

    def status(self, stream=None) -> int:
        return int(lib.rq_ctx_check(self._h, _stream(stream)))

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def default_launch(kind: int = CWBVH, query: int = ANY) -> Launch:
    l = Launch()
    check(lib.rq_default_launch(kind, query, C.byref(l)), "rq_default_launch")
    return l


# ------------------------------------------------------------ tracing ----

def trace(ctx: Context, scene: Scene, rays, hits, query: int = ANY, launch: Optional[Launch] = None,
          stream=None, count: Optional[int] = None) -> None:
    """Trace rays (CUDA tensor, 32 B per ray) into hits (16 B per ray)."""
    n = _rows(rays, 8, "rays") if count is None else count
    check(lib.rq_trace(ctx._h, scene._h, _ptr(rays), _ptr(hits), n, query,
                       C.byref(launch) if launch is not None else None, _stream(stream)), "rq_trace")


def trace_ordered(ctx: Context, scene: Scene, rays, hits, query: int = ANY, stream=None) -> None:
    """Trace in the oracle's traversal order (bit-identical results)."""
    check(lib.rq_trace_ordered(ctx._h, scene._h, _ptr(rays), _ptr(hits), _rows(rays, 8, "rays"), query,
                               _stream(stream)), "rq_trace_ordered")


def shard_range(count: int, n_parts: int, part: int):
    """(begin, size) of ray range `part` of `count` over `n_parts` (rq_shard_range)."""
    b, m = C.c_int64(), C.c_int64()
    check(lib.rq_shard_range(count, n_parts, part, C.byref(b), C.byref(m)), "rq_shard_range")
    return b.value, m.value


class Sharded:
    """One ray set over several devices holding replicas of one scene
    (rq_sharded_*): contiguous ray ranges per device, hits gathered into the
    caller's buffer on the first device by peer copies."""

    def __init__(self, devices: Sequence[int], scenes: Sequence["Scene"], max_rays: int):
        if len(devices) != len(scenes) or not devices:
            raise ValueError("one scene per device")
        self._scenes = list(scenes)
        devs = (C.c_int * len(devices))(*devices)
        hs = (C.c_void_p * len(scenes))(*[sc._h.value if isinstance(sc._h, C.c_void_p) else sc._h for sc in scenes])
        h = C.c_void_p()
        check(lib.rq_sharded_create(len(devices), devs, hs, max_rays, C.byref(h)), "rq_sharded_create")
        self._h = h

    def trace(self, rays, hits, query: int = ANY, launch: Optional[Launch] = None, stream=None) -> None:
        n = _rows(rays, 8, "rays")
        check(lib.rq_sharded_trace(self._h, _ptr(rays), _ptr(hits), n, query,
                                   C.byref(launch) if launch is not None else None, _stream(stream)),
              "rq_sharded_trace")

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib.rq_sharded_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Tlas:
    """Instances of CWBVH scenes under a top-level CWBVH (rq_tlas_*).

    transforms: (n, 3, 4) object-to-world affine matrices; blas_index: (n,)
    indices into `blas`.  The bottom-level scenes are kept alive here."""

    def __init__(self, blas: Sequence[Scene], transforms, blas_index):
        m = np.ascontiguousarray(transforms, np.float32).reshape(-1, 12)
        bi = np.ascontiguousarray(blas_index, np.int32).reshape(-1)
        if m.shape[0] != bi.size:
            raise ValueError("one transform per instance")
        self._blas = list(blas)
        arr = (C.c_void_p * len(self._blas))(*[b._h.value if isinstance(b._h, C.c_void_p) else b._h
                                                for b in self._blas])
        h = C.c_void_p()
        check(lib.rq_tlas_create(arr, len(self._blas), m.ctypes.data, bi.ctypes.data, bi.size, C.byref(h)),
              "rq_tlas_create")
        self._h = h
        self.n_instances = bi.size

    def buffers(self) -> dict:
        """Host copies of the top-level buffers (nodes, rows, map)."""
        n, nn, r, nr, mp = C.c_void_p(), C.c_int64(), C.c_void_p(), C.c_int64(), C.c_void_p()
        check(lib.rq_tlas_buffers(self._h, C.byref(n), C.byref(nn), C.byref(r), C.byref(nr), C.byref(mp)),
              "rq_tlas_buffers")
        f = lambda ptr, k, t: np.ctypeslib.as_array(C.cast(ptr, C.POINTER(t)), shape=(k,)).copy()  # noqa: E731
        return {"nodes": f(n, 4 * nn.value, C.c_float).reshape(-1, 4),
                "rows": f(r, 4 * nr.value, C.c_float).reshape(-1, 4),
                "map": f(mp, nr.value, C.c_int32)}

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_tlas_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def build_tlas_host(blas_bounds, transforms, blas_index) -> HostBVH:
    """The top-level tree alone, built on the host (rq_tlas_build_host):
    blas_bounds (n_blas, 6) lo/hi, transforms (n, 3, 4), blas_index (n,).
    The result's nodes / woop / prim_index are the top-level nodes, the
    instance rows and the (instance, blas, -1) map."""
    bb = np.ascontiguousarray(blas_bounds, np.float32).reshape(-1, 6)
    m = np.ascontiguousarray(transforms, np.float32).reshape(-1, 12)
    bi = np.ascontiguousarray(blas_index, np.int32).reshape(-1)
    if m.shape[0] != bi.size:
        raise ValueError("one transform per instance")
    h = C.c_void_p()
    check(lib.rq_tlas_build_host(bb.ctypes.data, bb.shape[0], m.ctypes.data, bi.ctypes.data, bi.size, C.byref(h)),
          "rq_tlas_build_host")
    hb = HostBVH.__new__(HostBVH)
    hb.vertices = hb.indices = None
    hb._adopt(h)
    hb.kind = CWBVH
    return hb


def trace_instanced(ctx: Context, tlas: Tlas, rays, hits, query: int = ANY, instance_out=None,
                    launch: Optional[Launch] = None, stream=None, ordered: bool = False) -> None:
    """Trace world-space rays through a Tlas; instance_out (int32, one per
    ray) receives the hit instance (-1 on a miss).  ordered=True turns
    postponing off: the oracle's traversal order, bit-identical results."""
    n = _rows(rays, 8, "rays")
    if ordered:
        launch = Launch(0, 0, 0, -1.0, 0, 0)
    check(lib.rq_trace_instanced(ctx._h, tlas._h, _ptr(rays), _ptr(hits),
                                 _ptr(instance_out) if instance_out is not None else None, n, query,
                                 C.byref(launch) if launch is not None else None, _stream(stream)),
          "rq_trace_instanced")


def trace_ao(ctx: Context, scene: Scene, rays, spp: int, occluded=None, launch: Optional[Launch] = None,
             stream=None):
    """Fused AO bake (rq_trace_ao): per-surfel occluded-ray counts (int32
    tensor, rays surfel-major with `spp` per surfel); AO = counts / spp.
    `occluded`, if given, is accumulated into."""
    import torch
    n = _rows(rays, 8, "rays")
    if spp <= 0 or n % spp:
        raise ValueError(f"{n} rays are not a whole number of surfels of {spp} rays")
    if occluded is None:
        with _On(stream):
            occluded = torch.zeros(n // spp, dtype=torch.int32, device=rays.device)
    check(lib.rq_trace_ao(ctx._h, scene._h, _ptr(rays), n, spp, _ptr(occluded),
                          C.byref(launch) if launch is not None else None, _stream(stream)), "rq_trace_ao")
    return occluded


def trace_counted(ctx: Context, scene: Scene, rays, hits, query: int = ANY, stream=None):
    """Trace and return per-ray (node fetches, triangle tests) as int32 tensors."""
    import torch
    n = _rows(rays, 8, "rays")
    with _On(stream):
        nv = torch.zeros(n, dtype=torch.int32, device=rays.device)
        nt = torch.zeros(n, dtype=torch.int32, device=rays.device)
    check(lib.rq_trace_counted(ctx._h, scene._h, _ptr(rays), _ptr(hits), n, query, _ptr(nv), _ptr(nt),
                               _stream(stream)), "rq_trace_counted")
    return nv, nt


def aorays(pos, nrm, radius, spp: int, seed: int = 0, tmin: float = 0.01, tmax: float = 1e20,
           offset_scale: float = 0.5, out=None, stream=None):
    """AO rays from a surfel cache (pos/nrm float4 tensors, radius float or None)."""
    import torch
    ns = _rows(pos, 4, "pos")
    if out is None:
        with _On(stream):
            out = torch.empty((ns * spp, 8), dtype=torch.float32, device=pos.device)
    check(lib.rq_aorays(_ptr(pos), _ptr(nrm), _ptr(radius) or None, ns, spp, seed, tmin, tmax, offset_scale,
                        _ptr(out), _stream(stream)), "rq_aorays")
    return out


def sample_surfels(vertices, indices, n: int, seed: int = 0, stream=None):
    """n surfels at uniform (triangle, barycentric) points of a device mesh."""
    import torch
    dev = vertices.device
    with _On(stream):
        pos = torch.empty((n, 4), dtype=torch.float32, device=dev)
        nrm = torch.empty((n, 4), dtype=torch.float32, device=dev)
        rad = torch.empty((n,), dtype=torch.float32, device=dev)
    nt = indices.numel() // 3
    check(lib.rq_sample_surfels(_ptr(vertices), _ptr(indices), nt, n, seed, _ptr(pos), _ptr(nrm), _ptr(rad),
                                _stream(stream)), "rq_sample_surfels")
    return pos, nrm, rad


def camera_rays(eye, look, up, vfov_deg: float, width: int, height: int, tmin: float = 0.0, tmax: float = 1e20,
                stream=None, tile: Optional[tuple] = None):
    """Pinhole camera rays, one per pixel (a torch CUDA (w*h, 8) tensor):
    row-major, or with tile=(tw, th) in tile order (rq_camera_rays_tiled)."""
    import torch
    with _On(stream):
        out = torch.empty((width * height, 8), dtype=torch.float32, device="cuda")
    f3 = lambda v: (C.c_float * 3)(*[float(x) for x in v])  # noqa: E731
    if tile is None:
        check(lib.rq_camera_rays(f3(eye), f3(look), f3(up), vfov_deg, width, height, tmin, tmax, _ptr(out),
                                 _stream(stream)), "rq_camera_rays")
    else:
        check(lib.rq_camera_rays_tiled(f3(eye), f3(look), f3(up), vfov_deg, width, height, int(tile[0]),
                                       int(tile[1]), tmin, tmax, _ptr(out), _stream(stream)), "rq_camera_rays_tiled")
    return out


def surfels_from_hits(rays, hits, scene: "Scene", stream=None):
    """Surfels at closest-hit points (facing geometric normals); misses get a zero normal."""
    import torch
    n = _rows(rays, 8, "rays")
    if _rows(hits, 4, "hits") < n:
        raise ValueError(f"hits: fewer than the {n} rows of rays")
    with _On(stream):
        pos = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        nrm = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        rad = torch.empty((n,), dtype=torch.float32, device="cuda")
    check(lib.rq_surfels_from_hits(scene._h, _ptr(rays), _ptr(hits), n, _ptr(pos), _ptr(nrm), _ptr(rad),
                                   _stream(stream)), "rq_surfels_from_hits")
    return pos, nrm, rad


def ao_reduce(hits, n_surfels: int, spp: int, stream=None):
    import torch
    with _On(stream):
        ao = torch.empty(n_surfels, dtype=torch.float32, device=hits.device)
    check(lib.rq_ao_reduce(_ptr(hits), n_surfels, spp, _ptr(ao), _stream(stream)), "rq_ao_reduce")
    return ao


def sort_rays(ctx: Context, rays, bounds_lo, bounds_hi, stream=None):
    import torch
    n = _rows(rays, 8, "rays")
    with _On(stream):
        out = torch.empty_like(rays)
        perm = torch.empty(n, dtype=torch.int32, device=rays.device)
    lo = (C.c_float * 3)(*bounds_lo)
    hi = (C.c_float * 3)(*bounds_hi)
    check(lib.rq_sort_rays(ctx._h, _ptr(rays), n, lo, hi, _ptr(out), _ptr(perm), _stream(stream)), "rq_sort_rays")
    return out, perm


def _items(items: Sequence[tuple]):
    arr = (N.BatchItem * len(items))()
    for k, (scene, rays, hits) in enumerate(items):
        arr[k] = N.BatchItem(scene._h, _ptr(rays), _ptr(hits), _rows(rays, 8, "rays"))
    return arr


class Batch:
    """Many (scene, rays, hits) items traced in one persistent launch."""

    def __init__(self, ctx: Context, items: Sequence[tuple], query: int = ANY, launch: Optional[Launch] = None,
                 sort_threshold: int = -1, use_graph: bool = False, params: Optional[N.BatchParams] = None):
        self._keep = list(items)
        arr = _items(items)
        if params is None:
            params = N.BatchParams(launch if launch is not None else Launch(), sort_threshold, int(use_graph))
        self.params = params
        h = C.c_void_p()
        check(lib.rq_batch_create(ctx._h, arr, len(items), query, C.byref(params), C.byref(h)), "rq_batch_create")
        self._h = h

    def run(self, stream=None) -> None:
        check(lib.rq_batch_run(self._h, _stream(stream)), "rq_batch_run")

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


def autotune(ctx: Context, scene: Scene, rays, hits, query: int = ANY, cache_path: Optional[str] = None,
             stream=None) -> Launch:
    l = Launch()
    check(lib.rq_autotune(ctx._h, scene._h, _ptr(rays), _ptr(hits), _rows(rays, 8, "rays"), query,
                          cache_path.encode() if cache_path else None, C.byref(l), _stream(stream)), "rq_autotune")
    return l


def autotune_batch(ctx: Context, items: Sequence[tuple], query: int = ANY, cache_path: Optional[str] = None,
                   stream=None) -> N.BatchParams:
    arr = _items(items)
    bp = N.BatchParams()
    check(lib.rq_autotune_batch(ctx._h, arr, len(items), query, cache_path.encode() if cache_path else None,
                                C.byref(bp), _stream(stream)), "rq_autotune_batch")
    return bp


# ------------------------------------------------------------ serving ----

class Server:
    """Continuous-batching AO bake server (see rq_server_* in include/rq.h)."""

    def __init__(self, hbm_budget_bytes: int, query: int = ANY, streams: int = 3, max_batch_rays: int = 0,
                 launch: Optional[Launch] = None):
        p = N.ServerParams(hbm_budget_bytes, max_batch_rays, streams, query,
                           launch if launch is not None else Launch())
        h = C.c_void_p()
        check(lib.rq_server_create(C.byref(p), C.byref(h)), "rq_server_create")
        self._h = h
        self._scenes = []

    def add_scene(self, scene: Scene) -> int:
        sid = C.c_int32()
        check(lib.rq_server_add_scene(self._h, scene._h, C.byref(sid)), "rq_server_add_scene")
        self._scenes.append(scene)
        return sid.value

    def submit(self, scene_id: int, host_rays: np.ndarray, host_hits: np.ndarray) -> int:
        """host_rays (n, 8) float32 and host_hits (n, 4) float32, kept alive by the caller until wait()."""
        t = C.c_uint64()
        n = host_rays.size // 8
        check(lib.rq_server_submit(self._h, scene_id, host_rays.ctypes.data, host_hits.ctypes.data, n, C.byref(t)),
              "rq_server_submit")
        return t.value

    def submit_bake(self, scene_id: int, pos: np.ndarray, nrm: np.ndarray, radius: Optional[np.ndarray],
                    spp: int, seed: int, tmin: float, tmax: float, offset_scale: float, host_ao: np.ndarray) -> int:
        """AO bake request: host surfels (pos, nrm (n, 4) float32, radius (n,)
        or None) in, host_ao (n,) float32 out (occluded / spp); all arrays
        kept alive by the caller until wait()."""
        n = pos.shape[0]
        if nrm.shape[0] != n or host_ao.size < n or (radius is not None and radius.size < n):
            raise ValueError("pos, nrm, radius and host_ao need one entry per surfel")
        t = C.c_uint64()
        check(lib.rq_server_submit_bake(self._h, scene_id, pos.ctypes.data, nrm.ctypes.data,
                                        radius.ctypes.data if radius is not None else None, n, spp, seed, tmin,
                                        tmax, offset_scale, host_ao.ctypes.data, C.byref(t)),
              "rq_server_submit_bake")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        st = N.RequestStats()
        s = lib.rq_server_wait(self._h, ticket, timeout_ms, C.byref(st))
        out = {f: getattr(st, f) for f, _ in N.RequestStats._fields_}
        out["status_name"] = N.STATUS.get(s, str(s))
        if s not in (0,):
            raise RQError(s, "rq_server_wait")
        return out

    def cancel(self, ticket: int) -> int:
        return int(lib.rq_server_cancel(self._h, ticket))

    def memory(self) -> dict:
        """Pool accounting (rq_server_memory): pool, in-use and peak bytes,
        admission waits, pieces queued, rays per launch."""
        m = N.ServerMemoryStats()
        check(lib.rq_server_memory(self._h, C.byref(m)), "rq_server_memory")
        return {f: getattr(m, f) for f, _ in N.ServerMemoryStats._fields_}

    def close(self) -> None:
        # `lib` is None once the interpreter is tearing modules down; the
        # process exit releases the handle then.
        if getattr(self, "_h", None) and lib is not None:
            lib.rq_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


# ------------------------------------------ reference-shaped entry points ----

def rtBindCWBVHData(nodes, woop, prim_index=None) -> None:
    check(lib.rq_rtBindCWBVHData(_ptr(nodes), _ptr(woop), _ptr(prim_index) or None), "rtBindCWBVHData")


def rtTraceCWBVH(rays, hits, ray_count: int) -> None:
    check(lib.rq_rtTraceCWBVH(_ptr(rays), _ptr(hits), ray_count), "rtTraceCWBVH")


def rtBindBVH2Data(nodes, woop, prim_index=None) -> None:
    check(lib.rq_rtBindBVH2Data(_ptr(nodes), _ptr(woop), _ptr(prim_index) or None), "rtBindBVH2Data")


def rtTraceBVH2(rays, hits, ray_count: int) -> None:
    check(lib.rq_rtTraceBVH2(_ptr(rays), _ptr(hits), ray_count), "rtTraceBVH2")


def rtOccludedCWBVH(rays, hits, ray_count: int) -> None:
    check(lib.rq_rtOccludedCWBVH(_ptr(rays), _ptr(hits), ray_count), "rtOccludedCWBVH")


def rtOccludedBVH2(rays, hits, ray_count: int) -> None:
    check(lib.rq_rtOccludedBVH2(_ptr(rays), _ptr(hits), ray_count), "rtOccludedBVH2")


def GenerateAORaysUniform(num_texels: int, rays_per_texel: int, pos: np.ndarray, nrm: np.ndarray,
                          radius: np.ndarray):
    """Host surfel arrays in, a torch CUDA tensor of rays out (tmin 0.01, tmax 1e20, offset radius/2)."""
    import torch
    pos = np.ascontiguousarray(pos, np.float32)
    nrm = np.ascontiguousarray(nrm, np.float32)
    radius = np.ascontiguousarray(radius, np.float32)
    p = lib.rq_GenerateAORaysUniform(num_texels, rays_per_texel, pos.ctypes.data, nrm.ctypes.data,
                                     radius.ctypes.data)
    if not p:
        raise RQError(5, "GenerateAORaysUniform")
    n = num_texels * rays_per_texel
    out = torch.empty((n, 8), dtype=torch.float32, device="cuda")
    try:
        check(lib.rq_device_copy(out.data_ptr(), p, n * 32), "rq_device_copy")
    finally:
        lib.rq_device_free(p)
    return out
