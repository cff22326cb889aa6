"""Scene and sample-cache files: the reference's mesh.dat / samplecache.dat
formats (src/main.cpp:31-45, :52-64) and the library's converted-scene file.

The files are written here independently with numpy in the layout the
reference's main() reads, then loaded through the C ABI; the library's own
writers must produce the same bytes.
"""
import numpy as np
import pytest


def _mesh_bytes(V, I, M):
    hdr = np.array([V.shape[0], I.shape[0]], np.int32).tobytes()
    return hdr + V.astype(np.float32).tobytes() + I.astype(np.int32).tobytes() + M.astype(np.int32).tobytes()


def _cache_bytes(sx, sy, P, Nn, R):
    return (np.array([sx, sy], np.int32).tobytes() + P.astype(np.float32).tobytes()
            + Nn.astype(np.float32).tobytes() + R.astype(np.float32).tobytes())


@pytest.fixture
def mesh(rq):
    V, I = rq.gen_heightfield_boxes(3, grid=16, n_boxes=20)
    M = (np.arange(I.shape[0]) % 5).astype(np.int32)
    return V, I, M


def test_mesh_dat_round_trip(rq, mesh, tmp_path):
    V, I, M = mesh
    f = tmp_path / "mesh.dat"
    f.write_bytes(_mesh_bytes(V, I, M))
    v, i, m = rq.load_mesh_dat(f)
    assert np.array_equal(v, V) and np.array_equal(i, I) and np.array_equal(m, M)
    g = tmp_path / "mine.dat"
    rq.save_mesh_dat(g, V, I, M)
    assert g.read_bytes() == f.read_bytes()
    rq.save_mesh_dat(g, V, I)  # materials default to 0
    assert (rq.load_mesh_dat(g)[2] == 0).all()


def test_mesh_dat_rejects_bad_files(rq, mesh, tmp_path):
    V, I, M = mesh
    good = _mesh_bytes(V, I, M)
    f = tmp_path / "bad.dat"
    for blob in (good[:-4], good + b"\0", good[:6], np.array([-1, 0], np.int32).tobytes()):
        f.write_bytes(blob)
        with pytest.raises(rq.RQError, match="INVALID_ARG"):
            rq.load_mesh_dat(f)
    I2 = I.copy()
    I2[5, 1] = V.shape[0]  # index out of range
    f.write_bytes(_mesh_bytes(V, I2, M))
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.load_mesh_dat(f)
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.save_mesh_dat(tmp_path / "x.dat", V, I2)
    with pytest.raises(rq.RQError, match="NOT_FOUND"):
        rq.load_mesh_dat(tmp_path / "missing.dat")


def test_empty_mesh_dat(rq, tmp_path):
    f = tmp_path / "empty.dat"
    f.write_bytes(np.array([0, 0], np.int32).tobytes())
    v, i, m = rq.load_mesh_dat(f)
    assert v.shape == (0, 3) and i.shape == (0, 3) and m.shape == (0,)


def test_samplecache_round_trip(rq, tmp_path):
    rng = np.random.default_rng(5)
    sx, sy = 13, 7
    P = rng.normal(size=(sx * sy, 4)).astype(np.float32)
    Nn = rng.normal(size=(sx * sy, 4)).astype(np.float32)
    R = rng.random(sx * sy).astype(np.float32)
    f = tmp_path / "samplecache.dat"
    f.write_bytes(_cache_bytes(sx, sy, P, Nn, R))
    gx, gy, p, n, r = rq.load_samplecache_dat(f)
    assert (gx, gy) == (sx, sy)
    assert np.array_equal(p, P) and np.array_equal(n, Nn) and np.array_equal(r, R)
    g = tmp_path / "mine.dat"
    rq.save_samplecache_dat(g, sx, sy, P, Nn, R)
    assert g.read_bytes() == f.read_bytes()
    f.write_bytes(_cache_bytes(sx, sy, P, Nn, R)[:-1])
    with pytest.raises(rq.RQError, match="INVALID_ARG"):
        rq.load_samplecache_dat(f)
    with pytest.raises(ValueError):
        rq.save_samplecache_dat(g, sx + 1, sy, P, Nn, R)


@pytest.mark.parametrize("kind", [0, 1], ids=["cwbvh", "bvh2"])
def test_scene_file_round_trip(rq, po, mesh, kind, tmp_path):
    V, I, _ = mesh
    hb = rq.HostBVH(V, I, kind)
    f = tmp_path / "scene.rqs"
    hb.save(f)
    lb = rq.HostBVH.load(f)
    assert lb.kind == kind
    assert np.array_equal(lb.nodes.view(np.uint32), hb.nodes.view(np.uint32))  # node words are bit fields
    assert np.array_equal(lb.woop.view(np.uint32), hb.woop.view(np.uint32))
    assert np.array_equal(lb.prim_index, hb.prim_index)
    for k in ("node_count", "leaf_count", "depth", "kind", "bounds_lo", "bounds_hi", "node_float4s"):
        assert lb.info[k] == hb.info[k], k
    with pytest.raises(rq.RQError, match="NOT_FOUND"):
        lb.tree()
    # the loaded buffers answer the same queries
    rng = np.random.default_rng(1)
    rays = np.zeros((2000, 8), np.float32)
    rays[:, 0:3] = rng.uniform(-0.2, 1.2, (2000, 3))
    d = rng.normal(size=(2000, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = 10.0
    a = po.trace(kind, hb.nodes, hb.woop, rays, False)
    b = po.trace(kind, lb.nodes, lb.woop, rays, False)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_scene_file_rejects_corruption(rq, mesh, tmp_path):
    V, I, _ = mesh
    hb = rq.HostBVH(V, I, rq.CWBVH)
    f = tmp_path / "scene.rqs"
    hb.save(f)
    blob = bytearray(f.read_bytes())
    for bad in (bytes(blob[:-1]), bytes(blob) + b"\0", b"NOTSCENE" + bytes(blob[8:])):
        f.write_bytes(bad)
        with pytest.raises(rq.RQError, match="BAD_SCENE"):
            rq.HostBVH.load(f)
    blob[200] ^= 0x01  # one payload bit: the checksum catches it
    f.write_bytes(bytes(blob))
    with pytest.raises(rq.RQError, match="BAD_SCENE"):
        rq.HostBVH.load(f)
    with pytest.raises(rq.RQError, match="NOT_FOUND"):
        rq.HostBVH.load(tmp_path / "missing.rqs")
