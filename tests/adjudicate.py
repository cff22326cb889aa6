"""Parity comparison of two hit buffers with FP64 adjudication.

Tolerance (from the parity contract): any-hit occlusion bits and closest-hit
primitive ids must be equal and t must agree within 1e-6 relative; every
disagreement must be explained, in double precision on the original
vertices, as a tie (both candidates' t within 1e-5 relative), a hit within
1e-5 (relative) of tmin or tmax, or a hit within 1e-5 of a triangle edge in
barycentric coordinates.
"""
from __future__ import annotations

import numpy as np

T_REL = 1e-6
ADJ = 1e-5


def prim_ids(hits: np.ndarray, prim_index: np.ndarray) -> np.ndarray:
    addr = np.ascontiguousarray(hits[:, 1]).view(np.int32)
    return np.where(addr >= 0, prim_index[np.maximum(addr, 0)], -1)


def _f64(po, ray, V, I, prim):
    t = I[prim]
    return po.tri_f64(ray, V[t[0]], V[t[1]], V[t[2]])


def _explained(po, ray, V, I, prims) -> bool:
    tmin, tmax = float(ray[3]), float(ray[7])
    ts = []
    for p in prims:
        if p < 0:
            continue
        t, u, v, det = _f64(po, ray, V, I, p)
        w = 1.0 - u - v
        if min(abs(u), abs(v), abs(w)) < ADJ:
            return True  # edge / vertex
        scale = max(abs(t), 1e-30)
        if abs(t - tmin) <= ADJ * max(scale, abs(tmin)) or abs(t - tmax) <= ADJ * max(scale, abs(tmax)):
            return True  # at the ends of the ray interval
        ts.append(t)
    if len(ts) == 2 and abs(ts[0] - ts[1]) <= ADJ * max(abs(ts[0]), abs(ts[1]), 1e-30):
        return True  # tie
    return False


def compare(po, rays, got, want, prim_index, V, I, any_hit: bool, exact: bool = False) -> dict:
    """Returns counts; raises AssertionError on an unexplained disagreement."""
    g_id = prim_ids(got, prim_index)
    w_id = prim_ids(want, prim_index)
    if any_hit:
        bad = np.nonzero((g_id >= 0) != (w_id >= 0))[0]
    else:
        bad = np.nonzero(g_id != w_id)[0]
    unexplained = [int(i) for i in bad if not _explained(po, rays[i], V, I, (int(g_id[i]), int(w_id[i])))]
    same = (g_id == w_id) & (g_id >= 0)
    if exact:
        rows = np.any(np.ascontiguousarray(got).view(np.uint32) != np.ascontiguousarray(want).view(np.uint32), axis=1)
        t_err = float(rows.sum())  # rows that differ in any bit
    else:
        denom = np.maximum(np.abs(want[same, 0]), 1e-30)
        t_err = float(np.max(np.abs(got[same, 0] - want[same, 0]) / denom)) if same.any() else 0.0
    out = {"rays": int(rays.shape[0]), "disagree": int(bad.size), "unexplained": len(unexplained),
           "t_max_rel": t_err, "hits": int((w_id >= 0).sum())}
    assert not unexplained, f"unexplained disagreements at rays {unexplained[:10]} ({out})"
    if exact:
        assert bad.size == 0 and t_err == 0.0, out
    elif not any_hit:
        assert t_err <= T_REL, out
    return out
