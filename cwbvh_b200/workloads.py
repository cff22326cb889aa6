"""Seeded synthetic workloads standing in for the reference's missing
mesh.dat / samplecache.dat (src/main.cpp:29-77).

  heightfield_boxes   64x64 heightfield (8,192 tris) + 200 boxes (2,400 tris)
  scene_of_size       the same family scaled to a triangle count (batched sets)
  batched_sizes       triangle and ray counts of the 64-scene batched workload
  city / large        the mid-size and large procedural scenes
  ao_rays             AO rays from surfels at uniform (triangle, barycentric)
                      points, cosine-weighted about the geometric normal,
                      tmin = 1e-4 * diag, tmax = tmax_scale * diag

Scene seed s, ray seed s + 1000.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

import cwbvh_b200 as rq


def heightfield_boxes(seed: int = 0, grid: int = 64, n_boxes: int = 200):
    return rq.gen_heightfield_boxes(seed, grid, n_boxes, 0.01, 0.1)


def scene_of_size(seed: int, target_tris: int):
    """Heightfield + boxes with the 8192:2400 split of the small scene."""
    box_tris = int(round(target_tris * 2400 / 10592))
    n_boxes = max(1, box_tris // 12)
    grid = max(2, int(round(math.sqrt(max(2, target_tris - 12 * n_boxes) / 2))))
    return rq.gen_heightfield_boxes(seed, grid, n_boxes, 0.01, 0.1)


def diag(vertices: np.ndarray) -> float:
    return float(np.linalg.norm(vertices.max(0) - vertices.min(0)))


@dataclass
class DeviceScene:
    kind: int
    host: "rq.HostBVH"
    scene: "rq.Scene"
    vertices: object  # torch CUDA (nv, 3) float32
    indices: object   # torch CUDA (nt, 3) int32
    diag: float
    n_tris: int


def upload(vertices: np.ndarray, indices: np.ndarray, kind: int = rq.CWBVH, threads: int = 0) -> DeviceScene:
    import torch
    hb = rq.HostBVH(vertices, indices, kind, threads=threads)
    sc = rq.Scene.from_host(hb)
    v = torch.from_numpy(np.ascontiguousarray(vertices, np.float32)).cuda()
    i = torch.from_numpy(np.ascontiguousarray(indices, np.int32)).cuda()
    return DeviceScene(kind, hb, sc, v, i, diag(vertices), int(indices.shape[0]))


def ao_rays(ds: DeviceScene, n_rays: int, seed: int, tmax_scale: float = 0.1, spp: int = 1, stream=None):
    """n_rays AO rays (torch CUDA (n, 8) float32), surfel-major with spp rays per surfel."""
    n_surf = (n_rays + spp - 1) // spp
    pos, nrm, rad = rq.sample_surfels(ds.vertices, ds.indices, n_surf, seed, stream=stream)
    rays = rq.aorays(pos, nrm, rad, spp, seed + 1, 1e-4 * ds.diag, tmax_scale * ds.diag, 0.0, stream=stream)
    return rays[:n_rays].contiguous() if rays.shape[0] != n_rays else rays


def log_uniform(rng: np.random.Generator, lo: float, hi: float, n: int) -> np.ndarray:
    return np.exp(rng.uniform(math.log(lo), math.log(hi), n))


def batched_sizes(n: int = 64):
    """The batched workload's (triangles, rays) per scene: 64 draws from
    log-uniform [10k, 2M] triangles and [256K, 8M] rays (seed 12345), the
    first n of them; 19.1M triangles and 126.7M rays over all 64."""
    rng = np.random.default_rng(12345)
    tris = np.exp(rng.uniform(math.log(10_000), math.log(2_000_000), 64)).astype(np.int64)[:n]
    rays = np.exp(rng.uniform(math.log(256 * 1024), math.log(8 * 1024 * 1024), 64)).astype(np.int64)[:n]
    return tris, rays
