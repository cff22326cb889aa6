"""ctypes access to the checkers -- TEST INFRASTRUCTURE ONLY.

liboracle.so (oracle.c) is the CPU restatement of the reference's path;
_ref/libref.so is the reference's own code compiled from its sources (see
Makefile).  Only tests, __graft_entry__.smoke() and bench.py's CPU-baseline
leg use this module; the product package never imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_oracle = None
_ref = None

i64, i32, vp = C.c_int64, C.c_int32, C.c_void_p


def oracle():
    global _oracle
    if _oracle is None:
        p = HERE / "liboracle.so"
        if not p.exists():
            raise FileNotFoundError(f"{p} missing: run `make -C oracle`")
        lib = C.CDLL(str(p))
        lib.oracle_trace.restype = C.c_int
        lib.oracle_trace.argtypes = [C.c_int, vp, i64, vp, i64, vp, i64, C.c_int, vp, vp, vp, C.c_int]
        lib.oracle_tri_f64.restype = None
        lib.oracle_tri_f64.argtypes = [vp, vp, vp, vp, vp]
        lib.oracle_aorays.restype = None
        lib.oracle_aorays.argtypes = [vp, vp, vp, i64, C.c_int, C.c_uint64, C.c_float, C.c_float, C.c_float, vp]
        lib.oracle_philox.restype = None
        lib.oracle_philox.argtypes = [vp, C.c_uint32, C.c_uint32, vp]
        lib.oracle_max_threads.restype = C.c_int
        lib.oracle_trace_instanced.restype = C.c_int
        lib.oracle_trace_instanced.argtypes = [vp, i64, vp, i64, vp, C.c_int, vp, vp, vp, vp, vp, i64, C.c_int, vp,
                                               vp, C.c_int]
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return (HERE / "_ref" / "libref.so").exists()


def ref():
    global _ref
    if _ref is None:
        p = HERE / "_ref" / "libref.so"
        if not p.exists():
            raise FileNotFoundError(f"{p} missing: run `make -C oracle` where the reference tree exists")
        lib = C.CDLL(str(p))
        lib.ref_convert.restype = C.c_int
        lib.ref_convert.argtypes = [C.c_int, i64, vp, vp, vp, vp, vp, C.c_int, vp, vp,
                                    C.POINTER(vp), C.POINTER(i64), C.POINTER(vp), C.POINTER(i64),
                                    C.POINTER(vp), C.POINTER(i64)]
        lib.ref_free.argtypes = [vp]
        lib.ref_woopify.argtypes = [vp, vp, vp, vp]
        for name in ("ref_bind_cwbvh", "ref_bind_bvh2"):
            getattr(lib, name).argtypes = [vp, vp, vp]
        for name in ("ref_trace_cwbvh", "ref_trace_bvh2"):
            getattr(lib, name).argtypes = [vp, vp, C.c_int]
        lib.ref_aorays.restype = vp
        lib.ref_aorays.argtypes = [C.c_int, C.c_int, vp, vp, vp]
        lib.ref_cuda_free.argtypes = [vp]
        lib.ref_trace_cwbvh_grid.restype = C.c_int
        lib.ref_trace_cwbvh_grid.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.POINTER(C.c_int)]
        lib.ref_sync.restype = C.c_int
        _ref = lib
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def trace(kind: int, nodes: np.ndarray, woop: np.ndarray, rays: np.ndarray, any_hit: bool, threads: int = 0,
          counts: bool = False):
    """CPU traversal; returns hits (n, 4) float32 [and node visits, tri tests]."""
    nodes = np.ascontiguousarray(nodes, np.float32)
    woop = np.ascontiguousarray(woop, np.float32)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 4), np.float32)
    nv = np.zeros(n, np.int32) if counts else None
    nt = np.zeros(n, np.int32) if counts else None
    err = oracle().oracle_trace(kind, _p(nodes), nodes.size // 4, _p(woop) if woop.size else None, woop.size // 4,
                                _p(rays), n, int(any_hit), _p(hits), _p(nv) if counts else None,
                                _p(nt) if counts else None, threads)
    if err:
        raise RuntimeError(f"oracle traversal error bits {err}")
    return (hits, nv, nt) if counts else hits


def trace_instanced(tlas: dict, blas: list, rays: np.ndarray, any_hit: bool, threads: int = 0):
    """CPU two-level traversal.  tlas: {"nodes", "rows", "map"} host arrays
    (the library's top-level buffers); blas: [(nodes, woop), ...] of the
    bottom-level CWBVHs.  Returns (hits (n, 4) float32, instance (n,) int32)."""
    tn = np.ascontiguousarray(tlas["nodes"], np.float32)
    tr = np.ascontiguousarray(tlas["rows"], np.float32)
    tm = np.ascontiguousarray(tlas["map"], np.int32)
    bn = [np.ascontiguousarray(n, np.float32) for n, _ in blas]
    bw = [np.ascontiguousarray(w, np.float32) for _, w in blas]
    nb = len(blas)
    bn_p = (C.c_void_p * nb)(*[_p(a) for a in bn])
    bw_p = (C.c_void_p * nb)(*[_p(a) for a in bw])
    bn_n = np.array([a.size // 4 for a in bn], np.int64)
    bw_n = np.array([a.size // 4 for a in bw], np.int64)
    rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
    n = rays.shape[0]
    hits = np.zeros((n, 4), np.float32)
    inst = np.zeros(n, np.int32)
    err = oracle().oracle_trace_instanced(_p(tn), tn.size // 4, _p(tr), tr.size // 4, _p(tm), nb, bn_p, _p(bn_n),
                                          bw_p, _p(bw_n), _p(rays), n, int(any_hit), _p(hits), _p(inst), threads)
    if err:
        raise RuntimeError(f"oracle traversal error bits {err}")
    return hits, inst


def tri_f64(ray: np.ndarray, v0, v1, v2) -> np.ndarray:
    out = np.zeros(4, np.float64)
    r = np.ascontiguousarray(ray, np.float32)
    a, b, c = (np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2))
    oracle().oracle_tri_f64(_p(r), _p(a), _p(b), _p(c), _p(out))
    return out


def aorays(pos, nrm, radius, spp: int, seed: int, tmin: float, tmax: float, offset_scale: float) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.float32)
    nrm = np.ascontiguousarray(nrm, np.float32)
    rad = None if radius is None else np.ascontiguousarray(radius, np.float32)
    ns = pos.shape[0]
    out = np.zeros((ns * spp, 8), np.float32)
    oracle().oracle_aorays(_p(pos), _p(nrm), _p(rad) if rad is not None else None, ns, spp, seed, tmin, tmax,
                           offset_scale, _p(out))
    return out


def philox(ctr, key: int) -> np.ndarray:
    c = np.ascontiguousarray(ctr, np.uint32)
    out = np.zeros(4, np.uint32)
    oracle().oracle_philox(_p(c), key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF, _p(out))
    return out


def ref_convert(tree: dict, vertices: np.ndarray, indices: np.ndarray):
    """The reference converter on a builder tree -> (nodes, woop, prim_index)."""
    lib = ref()
    v = np.ascontiguousarray(vertices, np.float32)
    ix = np.ascontiguousarray(indices, np.int32)
    codes = np.ascontiguousarray(tree["codes"], np.int32)
    boxes = np.ascontiguousarray(tree["boxes"], np.float32)
    lf = np.ascontiguousarray(tree["leaf_first"], np.int32)
    lc = np.ascontiguousarray(tree["leaf_count"], np.int32)
    refs = np.ascontiguousarray(tree["prim_refs"], np.int32)
    on, ow, op = vp(), vp(), vp()
    nn, nw, npi = i64(), i64(), i64()
    rc = lib.ref_convert(tree["width"], codes.shape[0], _p(codes) if codes.size else None,
                         _p(boxes) if boxes.size else None, _p(lf) if lf.size else None,
                         _p(lc) if lc.size else None, _p(refs) if refs.size else None, int(tree["root_is_leaf"]),
                         _p(v), _p(ix), C.byref(on), C.byref(nn), C.byref(ow), C.byref(nw), C.byref(op),
                         C.byref(npi))
    if rc:
        raise RuntimeError("ref_convert failed")

    def take(ptr, n, dt):
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float if dt == np.float32 else C.c_int32)),
                                  shape=(max(n, 1),))[:n].copy()
        lib.ref_free(ptr)
        return a

    nodes = take(on, nn.value * 4, np.float32).reshape(-1, 4)
    woop = take(ow, nw.value * 4, np.float32).reshape(-1, 4)
    prim = take(op, npi.value, np.int32)
    return nodes, woop, prim


def ref_woopify(v0, v1, v2) -> np.ndarray:
    out = np.zeros(12, np.float32)
    a, b, c = (np.ascontiguousarray(x, np.float32) for x in (v0, v1, v2))
    ref().ref_woopify(_p(a), _p(b), _p(c), _p(out))
    return out.reshape(3, 4)
