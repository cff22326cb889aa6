"""Generates the golden fixtures under tests/golden/ from the reference's own
code (oracle/_ref/libref.so, compiled from the reference sources by
oracle/Makefile).  Run where the reference tree is present:

    make -C oracle && python tests/golden/make_golden.py [--traces]

convert_fixtures.npz  -- for a set of small scenes: the builder's tree (the
    input), and ConvertToGPUBVH2 / ConvertToGPUCompressedWideBVH output
    (nodes, Woop rows, primitive map) on that tree; plus WoopifyTriangle rows
    for sample and degenerate triangles.
trace_fixtures.npz (--traces, needs a GPU) -- rtTraceCWBVH / rtTraceBVH2
    closest-hit results of the reference kernels on a small scene and AO ray set.
"""
from __future__ import annotations

import argparse
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import cwbvh_b200 as rq  # noqa: E402
from cwbvh_b200 import workloads as W  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

OUT = Path(__file__).resolve().parent


def quads(n: int):
    tid = np.arange(n)
    V = np.zeros((3 * n, 3), np.float32)
    V[0::3] = np.stack([np.full(n, -1.1), np.full(n, -1.1), tid], 1)
    V[1::3] = np.stack([np.full(n, 1.1), np.full(n, -1.1), tid], 1)
    V[2::3] = np.stack([np.full(n, 1.1), np.full(n, 1.1), tid], 1)
    return V, np.arange(3 * n, dtype=np.int32).reshape(-1, 3)


def scenes():
    out = {}
    out["hfbox"] = W.heightfield_boxes(0, grid=24, n_boxes=40)
    V, I = W.heightfield_boxes(1, grid=16, n_boxes=0)
    V = V.copy()
    V[:, 2] = 0.0  # flat: zero z extent in every heightfield node
    out["flat"] = (V, I)
    out["quads"] = quads(100)
    out["one_tri"] = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.int32))
    out["city"] = rq.gen_city(3, 16)
    return out


def convert_fixtures():
    data = {}
    for name, (V, I) in scenes().items():
        data[f"{name}/V"] = V
        data[f"{name}/I"] = I
        for kind, tag in ((rq.CWBVH, "cw"), (rq.BVH2, "b2")):
            hb = rq.HostBVH(V, I, kind)
            tr = hb.tree()
            for k in ("codes", "boxes", "leaf_first", "leaf_count", "prim_refs"):
                data[f"{name}/{tag}/tree/{k}"] = tr[k]
            data[f"{name}/{tag}/tree/root_is_leaf"] = np.array(tr["root_is_leaf"])
            nodes, woop, prim = po.ref_convert(tr, V, I)
            data[f"{name}/{tag}/ref/nodes"] = nodes
            data[f"{name}/{tag}/ref/woop"] = woop
            data[f"{name}/{tag}/ref/prim"] = prim
    # Woopify on sample triangles, a degenerate one and axis-aligned ones.
    rng = np.random.default_rng(3)
    tris = rng.uniform(-2, 2, (64, 3, 3)).astype(np.float32)
    tris[0] = [[0, 0, 0], [1, 1, 1], [2, 2, 2]]      # collinear (degenerate)
    tris[1] = [[0, 0, 1], [1, 0, 1], [0, 1, 1]]      # in a z plane
    tris[2] = [[1, 0, 0], [1, 1, 0], [1, 0, 1]]      # in an x plane
    rows = np.stack([po.ref_woopify(t[0], t[1], t[2]) for t in tris])
    data["woopify/tris"] = tris
    data["woopify/ref_rows"] = rows
    np.savez_compressed(OUT / "convert_fixtures.npz", **data)
    print("wrote", OUT / "convert_fixtures.npz")


def trace_fixtures():
    import torch
    lib = po.ref()
    V, I = W.heightfield_boxes(0, grid=24, n_boxes=40)
    data = {"V": V, "I": I}
    ds = W.upload(V, I, rq.CWBVH)
    rays = W.ao_rays(ds, 8192, seed=1000)
    data["rays"] = rays.cpu().numpy()
    for kind, tag in ((rq.CWBVH, "cw"), (rq.BVH2, "b2")):
        hb = rq.HostBVH(V, I, kind)
        sc = rq.Scene.from_host(hb)
        import ctypes as C
        n, w, p = C.c_void_p(), C.c_void_p(), C.c_void_p()
        rq.check(rq.lib.rq_scene_device_buffers(sc._h, C.byref(n), C.byref(w), C.byref(p)), "buffers")
        hits = torch.full((rays.shape[0], 4), float("nan"), device="cuda")
        if kind == rq.CWBVH:
            lib.ref_bind_cwbvh(n, w, p)
            lib.ref_trace_cwbvh(rays.data_ptr(), hits.data_ptr(), rays.shape[0])
        else:
            lib.ref_bind_bvh2(n, w, p)
            lib.ref_trace_bvh2(rays.data_ptr(), hits.data_ptr(), rays.shape[0])
        torch.cuda.synchronize()
        data[f"{tag}/tree/codes"] = hb.tree()["codes"]
        data[f"{tag}/nodes"] = hb.nodes
        data[f"{tag}/woop"] = hb.woop
        data[f"{tag}/prim"] = hb.prim_index
        data[f"{tag}/ref_hits"] = hits.cpu().numpy()
    out = Path(sys.argv[sys.argv.index("--out") + 1]) if "--out" in sys.argv else OUT / "trace_fixtures.npz"
    np.savez_compressed(out, **data)
    print("wrote", out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--traces", action="store_true")
    ap.add_argument("--out")
    a = ap.parse_args()
    if a.traces:
        trace_fixtures()
    else:
        convert_fixtures()
