"""The C-ABI library: it loads, exports every entry point include/rq.h
declares (and the reference-signature C++ twins), and its host-only calls
and argument checks work without a GPU."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "rq.h"
LIB = ROOT / "cwbvh_b200" / "librq.so"


def declared():
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(rq_[A-Za-z0-9_]+)\s*\(", txt)))


def exported():
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_every_declared_symbol_is_exported():
    syms = exported()
    names = declared()
    assert len(names) > 50
    missing = [n for n in names if n not in syms]
    assert not missing, missing


def test_reference_signature_twins_exported():
    """C++-linkage functions with the reference's exact signatures
    (src/TraversalKernelCWBVH.h:3-11, src/TraversalKernelBVH2.h:3-11,
    src/ValidationKernels.h:3-9)."""
    syms = exported()
    for mangled in ("_Z15rtBindCWBVHDataPK6float4S1_PKi", "_Z12rtTraceCWBVHP3RayP3Hiti",
                    "_Z14rtBindBVH2DataPK6float4S1_PKi", "_Z11rtTraceBVH2P3RayP3Hiti",
                    "_Z21GenerateAORaysUniformiiP6float4S0_Pf"):
        assert mangled in syms, mangled


def test_library_has_no_oracle_dependency():
    """librq.so does not link or name the oracle."""
    out = subprocess.run(["ldd", str(LIB)], capture_output=True, text=True).stdout
    assert "oracle" not in out and "libref" not in out
    strings = subprocess.run(["strings", str(LIB)], capture_output=True, text=True).stdout
    assert "liboracle" not in strings and "oracle_trace" not in strings


def test_status_strings(rq):
    assert rq.lib.rq_status_string(0) == b"RQ_OK"
    assert rq.lib.rq_status_string(6) == b"RQ_ERR_BAD_SCENE"
    assert rq.version().startswith("rq ")


def test_host_build_and_info(rq):
    from cwbvh_b200 import workloads as W
    V, I = W.heightfield_boxes(0)
    assert V.shape == (65 * 65 + 8 * 200, 3) and I.shape == (10592, 3)
    hb = rq.HostBVH(V, I, rq.CWBVH)
    info = hb.info
    assert info["node_float4s"] == 5 * info["node_count"]
    # spatial splits (default budget 200 %) may store a triangle in several leaves
    assert 3 * I.shape[0] <= info["woop_float4s"] <= 9 * I.shape[0]
    assert info["prim_index_count"] == info["woop_float4s"]
    assert np.allclose(info["bounds_lo"], V.min(0)) and np.allclose(info["bounds_hi"], V.max(0))
    once = rq.HostBVH(V, I, rq.CWBVH, spatial_splits=-1).info
    assert once["woop_float4s"] == 3 * I.shape[0]
    hb2 = rq.HostBVH(V, I, rq.BVH2, spatial_splits=-1)
    assert hb2.info["node_float4s"] == 4 * hb2.info["node_count"]
    assert hb2.info["woop_float4s"] == 3 * I.shape[0] + hb2.info["leaf_count"]


def test_invalid_arguments(rq):
    import ctypes as C
    V = np.zeros((3, 3), np.float32)
    bad = np.array([[0, 1, 5]], np.int32)  # vertex index out of range
    h = C.c_void_p()
    assert rq.lib.rq_build_bvh(V.ctypes.data, 3, bad.ctypes.data, 1, 0, None, C.byref(h)) == 1
    assert rq.lib.rq_build_bvh(V.ctypes.data, 3, bad.ctypes.data, 1, 7, None, C.byref(h)) == 1
    assert rq.lib.rq_trace(None, None, None, None, 0, 0, None, None) == 1
    assert rq.lib.rq_scene_create(0, None, 0, None, 0, None, 0, 1, C.byref(h)) == 1
    assert rq.lib.rq_batch_create(None, None, 0, 0, None, C.byref(h)) == 1
    assert rq.lib.rq_server_create(None, C.byref(h)) == 1
    assert rq.lib.rq_aorays(None, None, None, -1, 1, 0, 0.0, 1.0, 0.0, None, None) == 1


def test_scene_generators_deterministic(rq):
    a = rq.gen_heightfield_boxes(5, 32, 50)
    b = rq.gen_heightfield_boxes(5, 32, 50)
    c = rq.gen_heightfield_boxes(6, 32, 50)
    assert np.array_equal(a[0], b[0]) and not np.array_equal(a[0], c[0])
    V, I = rq.gen_city(1, 100)
    assert I.shape[0] > 100 * 40 and (I < V.shape[0]).all()
    V, I = rq.gen_spheres_terrain(1, 200_000)
    assert 150_000 < I.shape[0] < 260_000


def test_no_device_errors_cleanly(rq):
    """Without a CUDA device the device calls return an error status."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    import ctypes as C
    h = C.c_void_p()
    st = rq.lib.rq_ctx_create(C.byref(h))
    assert st in (5, 10)  # RQ_ERR_CUDA or RQ_ERR_NO_DEVICE


def test_header_compiles_and_links_from_c(tmp_path):
    """include/rq.h is plain C: a C11 program includes it with every warning
    as an error, links against librq.so and runs the host-only entry points
    (build a BVH over two triangles, read its info, free it)."""
    import shutil
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "t.c"
    src.write_text(r'''
#include <stdio.h>
#include "rq.h"
int main(void) {
    const float v[12] = {0, 0, 0, 1, 0, 0, 0, 1, 0, 1, 1, 0};
    const int32_t idx[6] = {0, 1, 2, 1, 3, 2};
    rq_host_bvh_t hb = NULL;
    rq_build_params bp = {0};
    bp.spatial_splits = -1;
    if (rq_build_bvh(v, 4, idx, 2, RQ_BVH_CWBVH, &bp, &hb) != RQ_OK) return 1;
    rq_bvh_info info;
    if (rq_host_bvh_info(hb, &info) != RQ_OK) return 2;
    printf("%lld %lld %s\n", (long long)info.node_count, (long long)info.woop_float4s, rq_status_string(RQ_OK));
    rq_host_bvh_free(hb);
    return info.woop_float4s == 6 ? 0 : 3;
}
''')
    exe = tmp_path / "t"
    inc = ROOT / "include"
    subprocess.run([cc, "-std=c11", "-Wall", "-Wextra", "-Werror", "-pedantic", f"-I{inc}", str(src), "-o", str(exe),
                    str(LIB), f"-Wl,-rpath,{LIB.parent}"], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, (out.returncode, out.stdout, out.stderr)
    assert out.stdout.split()[-1] == "RQ_OK"
