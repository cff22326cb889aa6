// Drop-in adapters with the reference's host entry points.
//
// rtBindCWBVHData / rtTraceCWBVH      src/TraversalKernelCWBVH.h:3-11
// rtBindBVH2Data  / rtTraceBVH2       src/TraversalKernelBVH2.h:3-11
// GenerateAORaysUniform               src/ValidationKernels.h:3-9
//
// As in the reference there is one bound scene per BVH kind (the reference
// keeps the pointers in __device__ globals set by cudaMemcpyToSymbol,
// src/TraversalKernelCWBVH.cu:14-16,377-385), tracing is synchronous on the
// legacy default stream, and the buffers stay owned by the caller.  The bind
// calls take no sizes, so the extent of each buffer is read from its CUDA
// allocation (cuMemGetAddressRange); the kernels bounds-check against it.
//
// Two flavours are exported: extern "C" rq_* functions returning rq_status,
// and C++-linkage functions with the exact reference signatures, which --
// like the reference's cudaCheck (src/CUDAAssert.h:5-12) -- log and abort on
// an error.
#include <cuda.h>

#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "runtime.h"

namespace {

std::mutex g_mu;
rq_ctx* g_ctx = nullptr;
rq_scene g_bound[2];
bool g_has[2] = {false, false};

typedef CUresult (*GetRangeFn)(CUdeviceptr*, size_t*, CUdeviceptr);

// Bytes from p to the end of the CUDA allocation that contains it (0 if unknown).
int64_t bytes_to_allocation_end(const void* p) {
    static GetRangeFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuMemGetAddressRange", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (GetRangeFn)f;
    }
    if (!fn || !p) return 0;
    CUdeviceptr base = 0;
    size_t size = 0;
    if (fn(&base, &size, (CUdeviceptr)p) != CUDA_SUCCESS) return 0;
    return (int64_t)(base + size - (CUdeviceptr)p);
}

rq_status ensure_ctx() {
    if (g_ctx) return RQ_OK;
    return rq_ctx_create(&g_ctx);
}

rq_status bind(rq_bvh_kind kind, const void* nodes, const void* woop, const int32_t* prim) {
    if (!nodes || !woop) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    rq_status st = ensure_ctx();
    if (st != RQ_OK) return st;
    const int64_t nb = bytes_to_allocation_end(nodes), wb = bytes_to_allocation_end(woop);
    if (nb < 16 || wb < 16) return RQ_ERR_INVALID_ARG;
    rq_scene& sc = g_bound[kind];
    sc = rq_scene();
    sc.kind = kind;
    sc.nodes = (const float4*)nodes;
    sc.woop = (const float4*)woop;
    sc.prim_index = prim;
    sc.node_f4 = std::min<int64_t>(nb / 16, UINT32_MAX);
    sc.woop_f4 = std::min<int64_t>(wb / 16, UINT32_MAX);
    sc.owned = false;
    g_has[kind] = true;
    return RQ_OK;
}

rq_status trace_sync(rq_bvh_kind kind, rq_query q, void* rays, void* hits, int count) {
    if (count < 0 || (count > 0 && (!rays || !hits))) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_has[kind]) return RQ_ERR_NOT_FOUND;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const bool log = std::getenv("RQ_LOG") != nullptr;
    if (log) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
    }
    rq_status st = rq_trace(g_ctx, &g_bound[kind], (const rq_ray*)rays, (rq_hit*)hits, count, q, nullptr, nullptr);
    if (st == RQ_OK) st = rq_ctx_check(g_ctx, nullptr);
    if (log) {
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        std::printf("%.3fMS, %.2fMRays/s (rq %s %s)\n", ms, (double)count / 1e6 / (ms / 1e3),
                    kind == RQ_BVH_CWBVH ? "CWBVH" : "BVH2", q == RQ_ANY ? "any-hit" : "closest-hit");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return st;
}

void check_or_abort(rq_status st, const char* what) {
    if (st == RQ_OK) return;
    std::fprintf(stderr, "%s: %s %s\n", what, rq_status_string(st), rq_last_error());
    std::abort();
}

}  // namespace

extern "C" {

rq_status rq_rtBindCWBVHData(const void* nodes, const void* woop, const int32_t* prim_index) {
    return bind(RQ_BVH_CWBVH, nodes, woop, prim_index);
}
rq_status rq_rtTraceCWBVH(void* rays, void* hits, int ray_count) {
    return trace_sync(RQ_BVH_CWBVH, RQ_CLOSEST, rays, hits, ray_count);
}
rq_status rq_rtBindBVH2Data(const void* nodes, const void* woop, const int32_t* prim_index) {
    return bind(RQ_BVH_BVH2, nodes, woop, prim_index);
}
rq_status rq_rtTraceBVH2(void* rays, void* hits, int ray_count) {
    return trace_sync(RQ_BVH_BVH2, RQ_CLOSEST, rays, hits, ray_count);
}
rq_status rq_rtOccludedCWBVH(void* rays, void* hits, int ray_count) {
    return trace_sync(RQ_BVH_CWBVH, RQ_ANY, rays, hits, ray_count);
}
rq_status rq_rtOccludedBVH2(void* rays, void* hits, int ray_count) {
    return trace_sync(RQ_BVH_BVH2, RQ_ANY, rays, hits, ray_count);
}

void* rq_GenerateAORaysUniform(int num_texels, int rays_per_texel, const float* pos, const float* nrm,
                               const float* radius) {
    if (num_texels < 0 || rays_per_texel <= 0 || (num_texels > 0 && (!pos || !nrm || !radius))) return nullptr;
    const size_t n = (size_t)num_texels;
    void *dp = nullptr, *dn = nullptr, *dr = nullptr, *rays = nullptr;
    bool ok = cudaMalloc(&rays, std::max<size_t>(1, n * rays_per_texel) * sizeof(rq::Ray)) == cudaSuccess;
    ok = ok && cudaMalloc(&dp, std::max<size_t>(1, n) * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&dn, std::max<size_t>(1, n) * 16) == cudaSuccess;
    ok = ok && cudaMalloc(&dr, std::max<size_t>(1, n) * 4) == cudaSuccess;
    ok = ok && (n == 0 || cudaMemcpy(dp, pos, n * 16, cudaMemcpyHostToDevice) == cudaSuccess);
    ok = ok && (n == 0 || cudaMemcpy(dn, nrm, n * 16, cudaMemcpyHostToDevice) == cudaSuccess);
    ok = ok && (n == 0 || cudaMemcpy(dr, radius, n * 4, cudaMemcpyHostToDevice) == cudaSuccess);
    // The reference's fixed ray parameters: tmin 0.01, tmax 1e20, origin
    // offset radius / 2 (src/ValidationKernels.cu:97-100).
    ok = ok && rq_aorays((const float*)dp, (const float*)dn, (const float*)dr, (int64_t)n, rays_per_texel, 0, 0.01f,
                         1e20f, 0.5f, (rq_ray*)rays, nullptr) == RQ_OK;
    ok = ok && cudaDeviceSynchronize() == cudaSuccess;
    cudaFree(dp);
    cudaFree(dn);
    cudaFree(dr);
    if (!ok) {
        cudaFree(rays);
        return nullptr;
    }
    return rays;
}

}  // extern "C"

// C++-linkage twins with the reference's exact signatures (global Ray / Hit /
// float4 types), so a program compiled against the reference headers links
// against librq unchanged.
struct Ray;
struct Hit;

void rtBindCWBVHData(const float4* nodes, const float4* woop, const int* prim) {
    check_or_abort(rq_rtBindCWBVHData(nodes, woop, prim), "rtBindCWBVHData");
}
void rtTraceCWBVH(Ray* rays, Hit* hits, int count) { check_or_abort(rq_rtTraceCWBVH(rays, hits, count), "rtTraceCWBVH"); }
void rtBindBVH2Data(const float4* nodes, const float4* woop, const int* prim) {
    check_or_abort(rq_rtBindBVH2Data(nodes, woop, prim), "rtBindBVH2Data");
}
void rtTraceBVH2(Ray* rays, Hit* hits, int count) { check_or_abort(rq_rtTraceBVH2(rays, hits, count), "rtTraceBVH2"); }
Ray* GenerateAORaysUniform(int num_texels, int rays_per_texel, float4* pos, float4* nrm, float* radius) {
    void* r = rq_GenerateAORaysUniform(num_texels, rays_per_texel, (const float*)pos, (const float*)nrm, radius);
    if (!r) check_or_abort(RQ_ERR_CUDA, "GenerateAORaysUniform");
    return (Ray*)r;
}
