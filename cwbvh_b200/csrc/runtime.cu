// Contexts, device scenes and the plain trace entry points of the C ABI.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "host_common.h"
#include "runtime.h"

namespace rq {

static thread_local std::string g_last_error;

rq_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    cudaGetLastError();  // clear a sticky-free error so the next call starts clean
    if (e == cudaErrorMemoryAllocation) return RQ_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return RQ_ERR_NO_DEVICE;
    return RQ_ERR_CUDA;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

int device_sms(int device) {
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(device);
    if (it != cache.end()) return it->second;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) sms = 0;
    cache[device] = sms;
    return sms;
}

rq_launch resolve_launch(rq_bvh_kind kind, rq_query q, const rq_launch* l) {
    rq_launch r{};
    r.block_size = 128;
    r.blocks_per_sm = 0;
    r.smem_stack = 8;
    r.postpone_ratio = kind == RQ_BVH_CWBVH ? 0.2f : 0.0f;
    // Dynamic fetch (src/TraversalKernelCWBVH.cu:366-367 uses Nd = 4, Nw = 16):
    // a warp leaves its traversal loop to refill once the idle lanes beyond
    // Nd per iteration add up to Nw.  Nd = 2, Nw = 8 measured best on B200
    // on the batched AO, city primary and 30M-triangle workloads (10-15 %
    // over refilling at the first idle lane, 3-5 % over the reference's).
    r.fetch_nd = 2;
    r.fetch_nw = 8;
    r.step_limit = kDefaultStepLimit;
    (void)q;
    if (l) {
        if (l->block_size > 0) r.block_size = l->block_size;
        if (l->blocks_per_sm > 0) r.blocks_per_sm = l->blocks_per_sm;
        if (l->smem_stack > 0) r.smem_stack = l->smem_stack;
        if (l->postpone_ratio > 0.f) r.postpone_ratio = l->postpone_ratio;
        if (l->postpone_ratio < 0.f) r.postpone_ratio = 0.f;  // negative: postponing off
        if (l->fetch_nd > 0) r.fetch_nd = l->fetch_nd;
        if (l->fetch_nd < 0) r.fetch_nd = 0;  // negative: no idle lanes tolerated
        if (l->fetch_nw > 0) r.fetch_nw = l->fetch_nw;
        if (l->step_limit > 0) r.step_limit = l->step_limit;
    }
    // Below 1, so the lanes still holding triangles always include enough of
    // the warp to go ahead instead of postponing again.
    r.postpone_ratio = std::min(r.postpone_ratio, 0.95f);
    r.block_size = std::max(32, std::min(512, (r.block_size + 31) / 32 * 32));
    r.smem_stack = smem_entries_of(r.smem_stack);
    return r;
}

// Occupancy of a kernel variant at a block size (cached; also raises the
// dynamic shared-memory limit of the variant once).
static int blocks_per_sm(TraceKernelFn fn, int block, size_t smem) {
    static std::mutex mu;
    static std::map<std::tuple<void*, int, size_t>, int> cache;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_tuple((void*)fn, block, smem);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    if (smem > 48 * 1024) cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, (const void*)fn, block, smem) != cudaSuccess) nb = 1;
    cache[key] = std::max(1, nb);
    return cache[key];
}

rq_status launch_trace(rq_bvh_kind kind, rq_query q, const rq_launch& l, bool multi, bool count,
                       const TraceParams& p, cudaStream_t s) {
    if (p.total_rays <= 0) return RQ_OK;
    int dev = 0;
    RQ_CUDA(cudaGetDevice(&dev));
    // Any-hit launches with many rays per thread take the ring-prefetching kernel.
    TraceKernelFn fn = nullptr;
    size_t smem = 0;
    int nb = 1;
    auto pick = [&](bool ring) {
        fn = trace_kernel(kind, q == RQ_ANY, l.smem_stack, multi, count, ring);
        smem = trace_smem_bytes(kind, smem_entries_of(l.smem_stack), l.block_size, ring);
        nb = blocks_per_sm(fn, l.block_size, smem);
        if (l.blocks_per_sm > 0) nb = std::min(nb, l.blocks_per_sm);
    };
    const bool ring = kind == RQ_BVH_CWBVH && !count && q == RQ_ANY;
    pick(ring);
    if (ring && p.total_rays < (multi ? kRingMinRaysPerThread : kRingMinRaysPerThreadSingle) * device_sms(dev) * nb *
                                   l.block_size)
        pick(false);
    int64_t grid = (int64_t)device_sms(dev) * nb;
    // No more warps than rays need.
    const int64_t warps_needed = (p.total_rays + 31) / 32;
    const int64_t blocks_needed = (warps_needed * 32 + l.block_size - 1) / l.block_size;
    grid = std::max<int64_t>(1, std::min(grid, blocks_needed));
    void* args[] = {(void*)&p};
    RQ_CUDA(cudaLaunchKernel((const void*)fn, dim3((unsigned)grid), dim3((unsigned)l.block_size), args, smem, s));
    return RQ_OK;
}

void warm_launch_cache(rq_bvh_kind kind, rq_query q, const rq_launch& l, bool multi, bool count) {
    for (int ring = 0; ring <= (kind == RQ_BVH_CWBVH && !count && q == RQ_ANY ? 1 : 0); ++ring) {
        TraceKernelFn fn = trace_kernel(kind, q == RQ_ANY, l.smem_stack, multi, count, ring != 0);
        blocks_per_sm(fn, l.block_size, trace_smem_bytes(kind, smem_entries_of(l.smem_stack), l.block_size, ring != 0));
    }
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) device_sms(dev);
}

rq_status reset_counter(rq_ctx* ctx, cudaStream_t s) {
    RQ_CUDA(cudaMemsetAsync(&ctx->scratch->ray_counter, 0, sizeof(unsigned long long), s));
    return RQ_OK;
}

TraceItem scene_item(const rq_scene* sc, const rq_ray* rays, rq_hit* hits, int64_t count) {
    TraceItem it{};
    it.nodes = sc->nodes;
    it.woop = sc->woop;
    it.rays = reinterpret_cast<const Ray*>(rays);
    it.hits = reinterpret_cast<Hit*>(hits);
    it.perm = nullptr;
    it.ray_begin = 0;
    it.count = count;
    it.node_f4 = (uint32_t)std::min<int64_t>(sc->node_f4, UINT32_MAX);
    it.woop_f4 = (uint32_t)std::min<int64_t>(sc->woop_f4, UINT32_MAX);
    return it;
}

TraceParams base_params(rq_ctx* ctx, const rq_launch& l) {
    TraceParams p{};
    p.scratch = ctx->scratch;
    p.postpone_ratio = l.postpone_ratio;
    p.fetch_nd = l.fetch_nd;
    p.fetch_nw = l.fetch_nw;
    p.bvh2_speculative = 1;
    p.step_limit = l.step_limit;
    return p;
}

// Bounds of a scene from its root node (CWBVH: p and 255 * 2^e per axis;
// BVH2: union of the two child boxes).
static void bounds_from_root(rq_scene* sc, const float* root) {
    if (sc->kind == RQ_BVH_CWBVH) {
        uint32_t ew;
        std::memcpy(&ew, &root[3], 4);
        for (int a = 0; a < 3; ++a) {
            const int e = (int)(int8_t)((ew >> (8 * a)) & 0xFFu);
            sc->lo[a] = root[a];
            sc->hi[a] = root[a] + 255.0f * std::ldexp(1.0f, e);
        }
    } else {
        const float* n = root;
        const float lo[3] = {std::fmin(n[0], n[4]), std::fmin(n[2], n[6]), std::fmin(n[8], n[10])};
        const float hi[3] = {std::fmax(n[1], n[5]), std::fmax(n[3], n[7]), std::fmax(n[9], n[11])};
        for (int a = 0; a < 3; ++a) { sc->lo[a] = lo[a]; sc->hi[a] = hi[a]; }
    }
}

}  // namespace rq

using namespace rq;

extern "C" {

const char* rq_last_error(void) { return g_last_error.c_str(); }

const char* rq_version(void) { return "rq 0.1 sm_100a"; }

rq_status rq_device_copy(void* dst, const void* src, int64_t bytes) {
    if (bytes < 0 || (bytes > 0 && (!dst || !src))) return RQ_ERR_INVALID_ARG;
    if (bytes > 0) RQ_CUDA(cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDeviceToDevice));
    return RQ_OK;
}

rq_status rq_device_free(void* p) {
    if (p) RQ_CUDA(cudaFree(p));
    return RQ_OK;
}

int rq_device_sm_count(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    return device_sms(dev);
}

rq_status rq_ctx_create(rq_ctx_t* out) {
    if (!out) return RQ_ERR_INVALID_ARG;
    rq_ctx* c = new rq_ctx();
    cudaError_t e = cudaGetDevice(&c->device);
    if (e == cudaSuccess) e = cudaMalloc(&c->scratch, sizeof(DevScratch));
    if (e == cudaSuccess) e = cudaMemset(c->scratch, 0, sizeof(DevScratch));
    if (e != cudaSuccess) {
        if (c->scratch) cudaFree(c->scratch);
        delete c;
        return cuda_fail(e, "rq_ctx_create");
    }
    *out = c;
    return RQ_OK;
}

rq_status rq_ctx_destroy(rq_ctx_t ctx) {
    if (!ctx) return RQ_ERR_INVALID_ARG;
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->temp) cudaFree(ctx->temp);
    delete ctx;
    return RQ_OK;
}

rq_status rq_ctx_check(rq_ctx_t ctx, void* stream) {
    if (!ctx) return RQ_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    RQ_CUDA(cudaStreamSynchronize(s));
    unsigned err = 0;
    RQ_CUDA(cudaMemcpy(&err, &ctx->scratch->error, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (err) RQ_CUDA(cudaMemset(&ctx->scratch->error, 0, sizeof(unsigned)));
    if (err & kErrBadScene) return RQ_ERR_BAD_SCENE;
    if (err & kErrStackOverflow) return RQ_ERR_STACK_OVERFLOW;
    if (err & kErrTimeout) return RQ_ERR_TIMEOUT;
    return RQ_OK;
}

rq_status rq_scene_create(rq_bvh_kind kind, const void* nodes, int64_t node_float4s, const void* woop,
                          int64_t woop_float4s, const int32_t* prim_index, int64_t prim_index_count,
                          int copy_from_host, rq_scene_t* out) {
    if (!out || !nodes || node_float4s <= 0 || woop_float4s < 0 || (woop_float4s > 0 && !woop)) return RQ_ERR_INVALID_ARG;
    if (kind != RQ_BVH_CWBVH && kind != RQ_BVH_BVH2) return RQ_ERR_INVALID_ARG;
    if (kind == RQ_BVH_CWBVH && node_float4s < 5) return RQ_ERR_INVALID_ARG;
    if (kind == RQ_BVH_BVH2 && node_float4s < 4) return RQ_ERR_INVALID_ARG;
    if (node_float4s > (int64_t)UINT32_MAX || woop_float4s > (int64_t)UINT32_MAX) return RQ_ERR_INVALID_ARG;
    rq_scene* sc = new rq_scene();
    sc->kind = kind;
    sc->node_f4 = node_float4s;
    sc->woop_f4 = woop_float4s;
    sc->prim_count = prim_index ? prim_index_count : 0;
    cudaGetDevice(&sc->device);
    float root[20];
    if (copy_from_host) {
        sc->owned = true;
        void *dn = nullptr, *dw = nullptr, *dp = nullptr;
        // 256 B of zero padding after each buffer: a kernel that loads the
        // float4s after a BVH2 leaf terminator (as the reference's does,
        // src/TraversalKernelBVH2.cu:128-133) stays inside the allocation.
        constexpr size_t kPad = 256;
        cudaError_t e = cudaMalloc(&dn, (size_t)node_float4s * 16 + kPad);
        if (e == cudaSuccess) e = cudaMalloc(&dw, (size_t)std::max<int64_t>(1, woop_float4s) * 16 + kPad);
        if (e == cudaSuccess) e = cudaMemset(dn, 0, (size_t)node_float4s * 16 + kPad);
        if (e == cudaSuccess) e = cudaMemset(dw, 0, (size_t)std::max<int64_t>(1, woop_float4s) * 16 + kPad);
        if (e == cudaSuccess && sc->prim_count > 0) e = cudaMalloc(&dp, (size_t)sc->prim_count * 4);
        if (e == cudaSuccess) e = cudaMemcpy(dn, nodes, (size_t)node_float4s * 16, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && woop_float4s > 0) e = cudaMemcpy(dw, woop, (size_t)woop_float4s * 16, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && sc->prim_count > 0)
            e = cudaMemcpy(dp, prim_index, (size_t)sc->prim_count * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(dn); cudaFree(dw); cudaFree(dp);
            delete sc;
            return cuda_fail(e, "rq_scene_create");
        }
        sc->nodes = (const float4*)dn;
        sc->woop = (const float4*)dw;
        sc->prim_index = (const int32_t*)dp;
        std::memcpy(root, nodes, sizeof(float) * (kind == RQ_BVH_CWBVH ? 20 : 16));
    } else {
        sc->nodes = (const float4*)nodes;
        sc->woop = (const float4*)woop;
        sc->prim_index = prim_index;
        cudaError_t e = cudaMemcpy(root, nodes, sizeof(float) * (kind == RQ_BVH_CWBVH ? 20 : 16), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            delete sc;
            return cuda_fail(e, "rq_scene_create");
        }
    }
    bounds_from_root(sc, root);
    *out = sc;
    return RQ_OK;
}

rq_status rq_scene_from_host_bvh(rq_host_bvh_t bvh, rq_scene_t* out) {
    if (!bvh || !out) return RQ_ERR_INVALID_ARG;
    rq_bvh_info info;
    rq_status st = rq_host_bvh_info(bvh, &info);
    if (st != RQ_OK) return st;
    const float *n, *w;
    const int32_t* p;
    rq_host_bvh_buffers(bvh, &n, &w, &p);
    st = rq_scene_create((rq_bvh_kind)info.kind, n, info.node_float4s, w, info.woop_float4s, p, info.prim_index_count,
                         1, out);
    if (st == RQ_OK) {
        for (int a = 0; a < 3; ++a) {
            (*out)->lo[a] = info.bounds_lo[a];
            (*out)->hi[a] = info.bounds_hi[a];
        }
    }
    return st;
}

rq_status rq_scene_destroy(rq_scene_t scene) {
    if (!scene) return RQ_ERR_INVALID_ARG;
    if (scene->owned) {
        cudaFree((void*)scene->nodes);
        cudaFree((void*)scene->woop);
        if (scene->prim_index) cudaFree((void*)scene->prim_index);
    }
    delete scene;
    return RQ_OK;
}

rq_status rq_scene_device_buffers(rq_scene_t scene, const void** nodes, const void** woop, const int32_t** prim_index) {
    if (!scene) return RQ_ERR_INVALID_ARG;
    if (nodes) *nodes = scene->nodes;
    if (woop) *woop = scene->woop;
    if (prim_index) *prim_index = scene->prim_index;
    return RQ_OK;
}

rq_status rq_scene_sizes(rq_scene_t scene, int64_t* node_float4s, int64_t* woop_float4s, int64_t* prim_index_count) {
    if (!scene) return RQ_ERR_INVALID_ARG;
    if (node_float4s) *node_float4s = scene->node_f4;
    if (woop_float4s) *woop_float4s = scene->woop_f4;
    if (prim_index_count) *prim_index_count = scene->prim_count;
    return RQ_OK;
}

int64_t rq_scene_bytes(rq_scene_t scene) {
    if (!scene) return 0;
    return scene->node_f4 * 16 + scene->woop_f4 * 16 + scene->prim_count * 4;
}

rq_status rq_default_launch(rq_bvh_kind kind, rq_query query, rq_launch* out) {
    if (!out) return RQ_ERR_INVALID_ARG;
    *out = resolve_launch(kind, query, nullptr);
    return RQ_OK;
}

static rq_status trace_impl(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits, int64_t count,
                            rq_query query, const rq_launch* launch, int32_t* nv, int32_t* nt, int speculative,
                            void* stream, uint32_t* ao_counts = nullptr, int ao_spp = 0) {
    if (!ctx || !scene || count < 0 || (count > 0 && (!rays || (!hits && !ao_counts)))) return RQ_ERR_INVALID_ARG;
    if (query != RQ_CLOSEST && query != RQ_ANY) return RQ_ERR_INVALID_ARG;
    if (((uintptr_t)rays | (uintptr_t)hits) & 15u) return RQ_ERR_INVALID_ARG;  // float4 records
    if (count == 0) return RQ_OK;
    const rq_launch l = resolve_launch(scene->kind, query, launch);
    TraceParams p = base_params(ctx, l);
    p.single = scene_item(scene, rays, hits, count);
    p.items = nullptr;
    p.n_items = 1;
    p.total_rays = count;
    p.node_visits = nv;
    p.tri_tests = nt;
    p.single.ao_counts = ao_counts;
    p.single.ao_spp = ao_spp;
    if (speculative >= 0) p.bvh2_speculative = speculative;
    cudaStream_t s = (cudaStream_t)stream;
    rq_status st = reset_counter(ctx, s);
    if (st != RQ_OK) return st;
    return launch_trace(scene->kind, query, l, false, nv != nullptr, p, s);
}

rq_status rq_trace(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits, int64_t count, rq_query query,
                   const rq_launch* launch, void* stream) {
    return trace_impl(ctx, scene, rays, hits, count, query, launch, nullptr, nullptr, -1, stream);
}

rq_status rq_trace_counted(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits, int64_t count,
                           rq_query query, int32_t* node_visits, int32_t* tri_tests, void* stream) {
    if (!node_visits || !tri_tests) return RQ_ERR_INVALID_ARG;
    rq_launch l{};
    l.postpone_ratio = -1.0f;  // the oracle's order, so the counts are comparable per ray
    return trace_impl(ctx, scene, rays, hits, count, query, &l, node_visits, tri_tests, 0, stream);
}

rq_status rq_trace_ao(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, int64_t count, int spp,
                      uint32_t* occluded, const rq_launch* launch, void* stream) {
    if (spp <= 0 || count < 0 || count % spp != 0 || (count > 0 && !occluded)) return RQ_ERR_INVALID_ARG;
    return trace_impl(ctx, scene, rays, nullptr, count, RQ_ANY, launch, nullptr, nullptr, -1, stream, occluded, spp);
}

// Trace with the traversal order of the CPU oracle: no triangle postponing
// (CWBVH) and no speculative leaf postponing (BVH2).  Results are then
// bit-identical to the oracle's; used by the parity tests.
rq_status rq_trace_ordered(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits, int64_t count,
                           rq_query query, void* stream) {
    rq_launch l{};
    l.postpone_ratio = -1.0f;
    return trace_impl(ctx, scene, rays, hits, count, query, &l, nullptr, nullptr, 0, stream);
}

}  // extern "C"
