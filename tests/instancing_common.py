"""Shared set-up of the instancing tests: a few bottom-level meshes, random
affine instances of them, the equivalent flattened world mesh and rays."""
import numpy as np


def rotation(axis, angle):
    axis = np.asarray(axis, np.float64)
    axis = axis / np.linalg.norm(axis)
    x, y, z = axis
    c, s = np.cos(angle), np.sin(angle)
    C = 1 - c
    return np.array([[c + x * x * C, x * y * C - z * s, x * z * C + y * s],
                     [y * x * C + z * s, c + y * y * C, y * z * C - x * s],
                     [z * x * C - y * s, z * y * C + x * s, c + z * z * C]])


def make_instances(rq, n_inst=300, seed=0):
    rng = np.random.default_rng(seed)
    meshes = [rq.gen_heightfield_boxes(1, grid=16, n_boxes=30), rq.gen_city(2, 16),
              rq.gen_heightfield_boxes(5, grid=8, n_boxes=5)]
    blas = [rq.HostBVH(V, I, rq.CWBVH) for V, I in meshes]
    M = np.zeros((n_inst, 3, 4), np.float32)
    bi = rng.integers(0, len(meshes), n_inst).astype(np.int32)
    for k in range(n_inst):
        R = rotation(rng.normal(size=3), rng.uniform(0, 2 * np.pi))
        S = np.diag(rng.uniform(0.5, 2.0, 3))
        ext = np.ptp(meshes[bi[k]][0], axis=0).max()
        M[k, :, :3] = (R @ S) / ext
        M[k, :, 3] = rng.uniform(-4, 4, 3)
    # flattened world mesh: triangle offset of each instance
    Vs, Is, off, nv = [], [], [], 0
    tri_off = np.zeros(n_inst, np.int64)
    t = 0
    for k in range(n_inst):
        V, I = meshes[bi[k]]
        W = (V.astype(np.float64) @ M[k, :, :3].astype(np.float64).T + M[k, :, 3]).astype(np.float32)
        Vs.append(W)
        Is.append(I + nv)
        nv += V.shape[0]
        tri_off[k] = t
        t += I.shape[0]
    flat = (np.concatenate(Vs), np.concatenate(Is).astype(np.int32))
    return meshes, blas, M, bi, flat, tri_off


def world_rays(n, seed, tmax=3.0):
    rng = np.random.default_rng(seed)
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-5, 5, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 1e-4
    rays[:, 7] = tmax
    return rays


def flat_ids(hits, inst, blas, bi, tri_off):
    """Flattened-mesh triangle id of each instanced hit (-1 on a miss)."""
    addr = np.ascontiguousarray(hits[:, 1]).view(np.int32)
    out = np.full(addr.shape, -1, np.int64)
    for i in np.nonzero(addr >= 0)[0]:
        k = int(inst[i])
        out[i] = tri_off[k] + int(blas[bi[k]].prim_index[addr[i]])
    return out
