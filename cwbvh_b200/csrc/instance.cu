// Two-level traversal: a top-level CWBVH over instances of bottom-level CWBVH
// scenes (BLAS), each placed by an affine object-to-world transform.
//
// The top-level tree uses the CWBVH node format unchanged; its leaf
// "triangles" are instances: the three float4 where a Woop triangle would sit
// hold the rows of the instance's world-to-object transform, and the
// primitive map holds (instance, BLAS index, -1) for them.  A ray entering an
// instance is transformed into object space (o' = W o, d' = W_lin d, so the
// ray parameter t is the same in both spaces), the BLAS is traversed with the
// ordinary node and Woop tests, and on leaving it the world ray is reloaded.
// The top level's pending node group and instance group are pushed before
// entering, so the stack below the entry mark is the top level's and the
// traversal order is fixed: that order is restated by the oracle
// (oracle_trace_instanced), which the kernel matches bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "host_common.h"
#include "runtime.h"
#include "trace_common.cuh"

namespace rq {

struct BlasDesc {
    const float4* nodes;
    const float4* woop;
    uint32_t node_f4;
    uint32_t woop_f4;
};

struct InstParams {
    const float4* tlas_nodes;
    const float4* tlas_rows;    // 3 float4 per instance slot: world-to-object rows
    const int32_t* tlas_map;    // (instance, blas, -1) per row
    uint32_t tlas_node_f4, tlas_rows_f4;
    const BlasDesc* blas;
    int n_blas;
    const Ray* rays;
    Hit* hits;
    int32_t* inst_out;          // per ray: instance of the hit, -1 on a miss (may be null)
    int64_t total_rays;
    DevScratch* scratch;
    float postpone_ratio;       // triangle / instance postponing (0: the oracle's order)
    int fetch_nd, fetch_nw;
    int step_limit;             // node visits per ray (both levels) before kErrTimeout
};

namespace {

constexpr int kInstStack = 64;  // entries per lane (shared + local)

// Node test of one CWBVH node for a ray (src/TraversalKernelCWBVH.cu:117-289):
// the next node group (child base, inner hit bits | imask) and triangle group.
__device__ __forceinline__ void cwbvh_visit(const float4* np, float ox, float oy, float oz, float idx_, float idy,
                                            float idz, unsigned octinv4, float tmin, float tmax, uint2& ng,
                                            uint2& tg) {
    const float4 n0 = ld_nc(np + 0), n1 = ld_nc(np + 1), n2 = ld_nc(np + 2);
    const float4 n3 = ld_nc(np + 3), n4 = ld_nc(np + 4);
    const unsigned ew = __float_as_uint(n0.w);
    const float adjx = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)(ew & 0xFFu) + 127)) << 23), idx_);
    const float adjy = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)((ew >> 8) & 0xFFu) + 127)) << 23), idy);
    const float adjz = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)((ew >> 16) & 0xFFu) + 127)) << 23), idz);
    const float orx = __fmul_rn(-__fsub_rn(ox, n0.x), idx_);
    const float ory = __fmul_rn(-__fsub_rn(oy, n0.y), idy);
    const float orz = __fmul_rn(-__fsub_rn(oz, n0.z), idz);
    const unsigned hitmask = cwbvh_hitmask(n1, n2, n3, n4, adjx, adjy, adjz, orx, ory, orz, idx_ < 0.f, idy < 0.f,
                                           idz < 0.f, octinv4, tmin, tmax);
    ng = make_uint2(__float_as_uint(n1.x), (hitmask & 0xFF000000u) | (ew >> 24));
    tg = make_uint2(__float_as_uint(n1.y), hitmask & 0x00FFFFFFu);
}

template <bool ANY, int SMEM>
__global__ void __launch_bounds__(128, 8) cwbvh_inst_kernel(const InstParams p) {
    extern __shared__ uint2 sstack[];
    constexpr int LOCAL = kInstStack - SMEM;
    uint2 lstack[LOCAL];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned tid = threadIdx.x;
    const unsigned B = blockDim.x;

    // current level: the top-level tree, or the BLAS of instance `cur_inst`
    const float4* nodes = p.tlas_nodes;
    const float4* woop = p.tlas_rows;
    uint32_t node_f4 = p.tlas_node_f4, woop_f4 = p.tlas_rows_f4;
    bool in_blas = false;
    int inst_sp = 0, cur_inst = -1;

    float ox = 0.f, oy = 0.f, oz = 0.f, dx = 0.f, dy = 0.f, dz = 0.f, tmin = 0.f, tmax = 0.f;
    float idx_ = 0.f, idy = 0.f, idz = 0.f;
    unsigned octinv = 0, octinv4 = 0;
    uint2 ng = make_uint2(0u, 0u), tg = make_uint2(0u, 0u);
    int sp = 0, hit_addr = -1, hit_inst = -1, steps = 0;
    int64_t ray = 0;
    float hu = 0.f, hv = 0.f;
    bool active = false, exhausted = false;

    auto push = [&](uint2 v) -> bool {
        if (sp < SMEM) sstack[(unsigned)sp * B + tid] = v;
        else if (sp < kInstStack) lstack[sp - SMEM] = v;
        else return false;
        ++sp;
        return true;
    };
    auto pop = [&]() -> uint2 {
        --sp;
        return sp < SMEM ? sstack[(unsigned)sp * B + tid] : lstack[sp - SMEM];
    };
    auto set_ray = [&](float4 o, float4 d) {
        ox = o.x; oy = o.y; oz = o.z;
        dx = d.x; dy = d.y; dz = d.z;
        idx_ = guarded_rcp(dx);
        idy = guarded_rcp(dy);
        idz = guarded_rcp(dz);
        octinv = 7u - (((dx < 0.f) ? 4u : 0u) | ((dy < 0.f) ? 2u : 0u) | ((dz < 0.f) ? 1u : 0u));
        octinv4 = octinv * 0x01010101u;
    };
    auto to_world = [&]() {
        in_blas = false;
        nodes = p.tlas_nodes; woop = p.tlas_rows; node_f4 = p.tlas_node_f4; woop_f4 = p.tlas_rows_f4;
        set_ray(__ldg(&p.rays[ray].origin_tmin), __ldg(&p.rays[ray].dir_tmax));
    };
    auto finish = [&](unsigned err) {
        if (err) {
            atomicOr(&p.scratch->error, err);
            hit_addr = -1;
            hit_inst = -1;
        }
        __stcs(&p.hits[ray].t_triId_u_v, make_float4(tmax, __int_as_float(hit_addr), hu, hv));
        if (p.inst_out) p.inst_out[ray] = hit_addr >= 0 ? hit_inst : -1;
        active = false;
    };

    for (;;) {
        const bool need = !active && !exhausted;
        const unsigned needm = __ballot_sync(kFullMask, need);
        if (needm) {
            const int leader = __ffs(needm) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&p.scratch->ray_counter, (unsigned long long)__popc(needm));
            base = __shfl_sync(kFullMask, base, leader);
            if (need) {
                const int64_t g = (int64_t)base + __popc(needm & lanemask_lt());
                if (g < p.total_rays) {
                    ray = g;
                    to_world();
                    tmin = __ldg(&p.rays[g].origin_tmin).w;
                    tmax = __ldg(&p.rays[g].dir_tmax).w;
                    ng = make_uint2(0u, 0x80000000u);
                    tg = make_uint2(0u, 0u);
                    sp = 0; inst_sp = 0; cur_inst = -1;
                    hit_addr = -1; hit_inst = -1; hu = 0.f; hv = 0.f; steps = 0;
                    active = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(kFullMask, active) == 0u) break;

        int lost = 0;
        for (;;) {
            // ---- node phase
            if (active) {
                unsigned fault = 0u;
                if (ng.y > 0x00FFFFFFu) {
                    const unsigned hitsm = ng.y;
                    const unsigned bit = highest_bit(hitsm);
                    const unsigned base = ng.x;
                    ng.y &= ~(1u << bit);
                    if (ng.y > 0x00FFFFFFu && !push(ng)) fault = kErrStackOverflow;
                    const unsigned slot = (bit - 24u) ^ octinv;
                    const unsigned ci = base + (unsigned)__popc(hitsm & ~(0xFFFFFFFFu << slot));
                    if (++steps > p.step_limit) fault |= kErrTimeout;
                    if ((uint64_t)ci * 5u + 5u > (uint64_t)node_f4) fault |= kErrBadScene;
                    if (!fault) cwbvh_visit(nodes + (size_t)ci * 5u, ox, oy, oz, idx_, idy, idz, octinv4, tmin, tmax,
                                            ng, tg);
                } else {
                    tg = ng;
                    ng = make_uint2(0u, 0u);
                }
                if (fault) finish(fault);
            }

            // ---- triangles (bottom level) or instances (top level) of the group,
            // warp-synchronous; postponed when few lanes have work (as the flat kernel)
            {
                const int total = __popc(__ballot_sync(kFullMask, active));
                const int threshold = (int)((float)total * p.postpone_ratio);
                for (;;) {
                    const bool want = active && tg.y != 0u;
                    const unsigned wm = __ballot_sync(kFullMask, want);
                    if (wm == 0u) break;
                    if (__popc(wm) < threshold) {
                        if (want && !push(tg)) finish(kErrStackOverflow);
                        break;
                    }
                    if (!want) continue;
                    const unsigned ti = highest_bit(tg.y);
                    const unsigned tri = tg.x * 3u + ti * 3u;
                    tg.y &= ~(1u << ti);
                    if ((uint64_t)tri + 3u > (uint64_t)woop_f4) {
                        finish(kErrBadScene);
                        continue;
                    }
                    const float4 r0 = ld_nc(woop + tri), r1 = ld_nc(woop + tri + 1), r2 = ld_nc(woop + tri + 2);
                    if (in_blas) {
                        float t, u, v;
                        if (woop_test(r0, r1, r2, ox, oy, oz, dx, dy, dz, tmin, tmax, t, u, v)) {
                            tmax = t;
                            hit_addr = (int)tri;
                            hit_inst = cur_inst;
                            hu = u;
                            hv = v;
                            if (ANY) finish(0u);
                        }
                        continue;
                    }
                    const int inst = __ldg(p.tlas_map + tri);
                    const int b = __ldg(p.tlas_map + tri + 1);
                    if (b < 0 || b >= p.n_blas) {
                        finish(kErrBadScene);
                        continue;
                    }
                    if ((ng.y > 0x00FFFFFFu && !push(ng)) || (tg.y != 0u && !push(tg))) {
                        finish(kErrStackOverflow);
                        continue;
                    }
                    inst_sp = sp;
                    in_blas = true;
                    cur_inst = inst;
                    // object-space ray: o' = W [o; 1], d' = W_lin d
                    const float4 o = make_float4(
                        __fmaf_rn(r0.z, oz, __fmaf_rn(r0.y, oy, __fmaf_rn(r0.x, ox, r0.w))),
                        __fmaf_rn(r1.z, oz, __fmaf_rn(r1.y, oy, __fmaf_rn(r1.x, ox, r1.w))),
                        __fmaf_rn(r2.z, oz, __fmaf_rn(r2.y, oy, __fmaf_rn(r2.x, ox, r2.w))), 0.f);
                    const float4 d = make_float4(
                        __fmaf_rn(r0.z, dz, __fmaf_rn(r0.y, dy, __fmul_rn(r0.x, dx))),
                        __fmaf_rn(r1.z, dz, __fmaf_rn(r1.y, dy, __fmul_rn(r1.x, dx))),
                        __fmaf_rn(r2.z, dz, __fmaf_rn(r2.y, dy, __fmul_rn(r2.x, dx))), 0.f);
                    set_ray(o, d);
                    const BlasDesc bd = p.blas[b];
                    nodes = bd.nodes; woop = bd.woop; node_f4 = bd.node_f4; woop_f4 = bd.woop_f4;
                    ng = make_uint2(0u, 0x80000000u);
                    tg = make_uint2(0u, 0u);
                }
            }

            // ---- leave a finished instance, then continue with the stack
            if (active && ng.y <= 0x00FFFFFFu) {
                if (in_blas && sp == inst_sp) to_world();
                if (sp > 0) ng = pop();
                else finish(0u);
            }
            const unsigned am = __ballot_sync(kFullMask, active);
            if (am == 0u) break;
            lost += 32 - __popc(am) - p.fetch_nd;
            if (lost >= p.fetch_nw) break;
        }
    }
}

}  // namespace
}  // namespace rq

using namespace rq;

struct rq_tlas {
    int device = 0;
    rq_scene_t top = nullptr;           // CWBVH over the instances (owned)
    HostBVH host;                       // host copy of the top-level buffers
    BlasDesc* d_blas = nullptr;         // device descriptors of the BLAS scenes
    int n_blas = 0;
    int64_t n_inst = 0;
};

extern "C" {

rq_status rq_tlas_create(const rq_scene_t* blas, int n_blas, const float* object_to_world, const int32_t* blas_index,
                         int64_t n_instances, rq_tlas_t* out) {
    if (!out || !blas || n_blas <= 0) return RQ_ERR_INVALID_ARG;
    for (int b = 0; b < n_blas; ++b)
        if (!blas[b] || blas[b]->kind != RQ_BVH_CWBVH) return RQ_ERR_INVALID_ARG;
    try {
        std::vector<float> bounds((size_t)n_blas * 6);
        for (int b = 0; b < n_blas; ++b)
            for (int a = 0; a < 3; ++a) {
                bounds[6 * b + a] = blas[b]->lo[a];
                bounds[6 * b + 3 + a] = blas[b]->hi[a];
            }
        std::unique_ptr<rq_tlas> t(new rq_tlas());
        cudaGetDevice(&t->device);
        t->n_blas = n_blas;
        t->n_inst = n_instances;
        rq_host_bvh_t hb = nullptr;
        rq_status st = rq_tlas_build_host(bounds.data(), n_blas, object_to_world, blas_index, n_instances, &hb);
        if (st != RQ_OK) return st;
        t->host = std::move(hb->b);
        rq_host_bvh_free(hb);
        st = rq_scene_create(RQ_BVH_CWBVH, t->host.nodes.data(), (int64_t)t->host.nodes.size() / 4, t->host.woop.data(),
                             (int64_t)t->host.woop.size() / 4, t->host.prim_index.data(),
                             (int64_t)t->host.prim_index.size(), 1, &t->top);
        if (st != RQ_OK) return st;
        std::vector<BlasDesc> desc((size_t)n_blas);
        for (int b = 0; b < n_blas; ++b)
            desc[(size_t)b] = BlasDesc{blas[b]->nodes, blas[b]->woop, (uint32_t)blas[b]->node_f4,
                                       (uint32_t)blas[b]->woop_f4};
        cudaError_t e = cudaMalloc(&t->d_blas, sizeof(BlasDesc) * (size_t)n_blas);
        if (e == cudaSuccess)
            e = cudaMemcpy(t->d_blas, desc.data(), sizeof(BlasDesc) * (size_t)n_blas, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            rq_scene_destroy(t->top);
            cudaFree(t->d_blas);
            return cuda_fail(e, "rq_tlas_create");
        }
        *out = t.release();
        return RQ_OK;
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}

rq_status rq_tlas_destroy(rq_tlas_t tlas) {
    if (!tlas) return RQ_ERR_INVALID_ARG;
    rq_status st = rq_scene_destroy(tlas->top);
    cudaError_t e = cudaFree(tlas->d_blas);
    delete tlas;
    if (st != RQ_OK) return st;
    return e == cudaSuccess ? RQ_OK : cuda_fail(e, "rq_tlas_destroy");
}

rq_status rq_tlas_buffers(rq_tlas_t tlas, const float** nodes, int64_t* node_float4s, const float** rows,
                          int64_t* row_float4s, const int32_t** map) {
    if (!tlas) return RQ_ERR_INVALID_ARG;
    if (nodes) *nodes = tlas->host.nodes.data();
    if (node_float4s) *node_float4s = (int64_t)tlas->host.nodes.size() / 4;
    if (rows) *rows = tlas->host.woop.data();
    if (row_float4s) *row_float4s = (int64_t)tlas->host.woop.size() / 4;
    if (map) *map = tlas->host.prim_index.data();
    return RQ_OK;
}

rq_status rq_trace_instanced(rq_ctx_t ctx, rq_tlas_t tlas, const rq_ray* rays, rq_hit* hits, int32_t* instance_out,
                             int64_t count, rq_query query, const rq_launch* launch, void* stream) {
    if (!ctx || !tlas || count < 0 || (count > 0 && (!rays || !hits))) return RQ_ERR_INVALID_ARG;
    if (((uintptr_t)rays | (uintptr_t)hits) & 15u) return RQ_ERR_INVALID_ARG;  // float4 records
    if (query != RQ_CLOSEST && query != RQ_ANY) return RQ_ERR_INVALID_ARG;
    if (count == 0) return RQ_OK;
    cudaStream_t s = (cudaStream_t)stream;
    rq_status st = reset_counter(ctx, s);
    if (st != RQ_OK) return st;
    InstParams p{};
    const rq_scene* top = tlas->top;
    p.tlas_nodes = top->nodes;
    p.tlas_rows = top->woop;
    p.tlas_map = top->prim_index;
    p.tlas_node_f4 = (uint32_t)top->node_f4;
    p.tlas_rows_f4 = (uint32_t)top->woop_f4;
    p.blas = tlas->d_blas;
    p.n_blas = tlas->n_blas;
    p.rays = (const Ray*)rays;
    p.hits = (Hit*)hits;
    p.inst_out = instance_out;
    p.total_rays = count;
    p.scratch = ctx->scratch;
    const rq_launch l = resolve_launch(RQ_BVH_CWBVH, query, launch);
    // Postponing is off unless asked for: on the instanced city it measured
    // 2 % slower than the oracle's order (instance entries are postponed too).
    p.postpone_ratio = launch && launch->postpone_ratio > 0.f ? l.postpone_ratio : 0.f;
    p.fetch_nd = l.fetch_nd;
    p.fetch_nw = l.fetch_nw;
    p.step_limit = l.step_limit;
    constexpr int kSmem = 8, kBlock = 128;
    void (*fn)(InstParams) = query == RQ_ANY ? cwbvh_inst_kernel<true, kSmem> : cwbvh_inst_kernel<false, kSmem>;
    const size_t smem = (size_t)kSmem * kBlock * sizeof(uint2);
    int per_sm = 0;
    RQ_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, smem));
    const int64_t blocks_needed = (count + kBlock - 1) / kBlock;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)device_sms(ctx->device) * std::max(1, per_sm),
                                                                  blocks_needed));
    fn<<<grid, kBlock, smem, s>>>(p);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

}  // extern "C"
