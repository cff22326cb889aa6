// Persistent trace kernels for sm_100a: the compressed 8-wide BVH (CWBVH) and
// the binary BVH (BVH2), closest-hit and any-hit, over one scene or over a
// batch of (scene, rays) items in one launch.
//
// Work distribution (both kernels).  One CTA per SM slot stays resident for the
// whole launch.  A warp hands rays to its idle lanes from one 64-bit global
// counter: the lanes that need a ray vote, one lane adds their count to the
// counter and broadcasts the old value (the reference's per-warp atomicAdd,
// src/TraversalKernelCWBVH.cu:56-87, written with __shfl_sync instead of a
// volatile shared word so it is correct under independent thread scheduling).
// A warp re-fills after the idle lanes have cost Nw lane-iterations beyond Nd
// (src/TraversalKernelCWBVH.cu:365-371).  Large CWBVH any-hit launches take
// their rays through a per-warp ring of prefetched rays instead (below).  Every vote is
// over the full warp and every loop is warp-uniform, so lanes never diverge
// around a collective.
//
// Safety.  A ray whose stack would overflow, whose node/triangle index falls
// outside the buffers, or that runs more than the step limit is finished as
// a miss and the context's error word records why; the kernel itself never
// reads outside the buffers it was given and never spins without a bound.
#include <cstdio>

#include "device_api.h"
#include "trace_common.cuh"

namespace rq {

constexpr int kStackTotal = 64;  // entries per lane (shared + local)

#ifdef RQ_MAXNREG
#define RQ_KERNEL_BOUNDS __maxnreg__(RQ_MAXNREG)  // register cap (occupancy experiments)
#define RQ_BVH2_BOUNDS __maxnreg__(RQ_MAXNREG)
#else
#define RQ_KERNEL_BOUNDS __launch_bounds__(512)
// The BVH2 kernel fits 56 registers without spilling (nine 128-thread blocks
// per SM instead of eight): closest-hit +2.3 %, any-hit unchanged on the
// small scene; 48 spills and loses 2 % any-hit.
#define RQ_BVH2_BOUNDS __maxnreg__(56)
#endif
constexpr uint32_t kBvh2Sentinel = 0x76543210u;  // src/TraversalKernelBVH2.cu:33

// ------------------------------------------------- per-warp ray prefetch --
//
// The CWBVH any-hit kernels of large launches (RING) take rays 32 at a time per
// warp (one counter add per 32 rays) into a ring of 64 slots per warp in
// shared memory: two halves, each filled by one cp.async group (every lane
// copies one ray's 32 bytes and notes its batch item).  A refill hands idle
// lanes the next slots in order; the ray loads of a half were issued a refill
// or more earlier and no longer stall the warp, and neither a counter add nor
// the item search sits on its path.  A half is refilled as soon as its last
// slot is handed out.  The last rays of a launch stay tied to the warp whose
// ring holds them, which costs a short launch more than the ring saves, so
// the ring is used from kRingMinRaysPerThread rays per thread of the grid up
// (batches) and from kRingMinRaysPerThreadSingle up (one scene, where no item
// search is saved): +2 % on a batch of 64 scenes with 127M AO rays, +1 % on
// 64 scenes with 16.8M rays, +1.6 % on one 29.6M-triangle scene with 64M AO
// rays (440 per thread), -0.5 % on one scene with 16.8M rays (110 per
// thread), -6 % on one scene with 1M rays (7 per thread).  Any-hit only:
// closest-hit batches measured 1 % slower with the ring.
constexpr unsigned kRingHalf = 32;  // rays per counter add
constexpr unsigned kRingSlots = 2 * kRingHalf;
// rays [64][2] float4, the two halves' first global ray index, items [64]
constexpr size_t kRingBytesPerWarp = kRingSlots * sizeof(Ray) + 2 * sizeof(int64_t) + kRingSlots * sizeof(int);
static_assert(kRingBytesPerWarp % 16 == 0, "ring keeps 16 B alignment");

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The batch item holding global ray g, searching forward from `hint` (the
// item of a smaller ray index taken by the same lane; -1 for none).
__device__ __forceinline__ int find_item(const TraceParams& p, int64_t g, int hint) {
    int lo = hint, hi = p.n_items - 1;
    if (lo < 0 || lo > hi || p.items[lo].ray_begin > g) lo = 0;
    if (lo < hi && p.items[lo + 1].ray_begin <= g) {
        ++lo;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (p.items[mid].ray_begin <= g) lo = mid; else hi = mid - 1;
        }
    }
    return lo;
}

// Resolves a global ray index to its item (batch) and loads the ray.
struct Lane {
    const float4* nodes;
    const float4* woop;
    int64_t out_idx;
    int64_t gidx;
    int item;  // batch item of the ray (its hit buffer or AO counters are read at the end)
    uint32_t node_f4, woop_f4;
};

// Points a lane at global ray g of batch item `item` (0 for a single scene)
// and returns the item.
template <bool MULTI>
__device__ __forceinline__ const TraceItem* set_lane(const TraceParams& p, int64_t g, int item, Lane& L) {
    const TraceItem* it = MULTI ? p.items + item : &p.single;
    const int64_t local = g - (MULTI ? it->ray_begin : 0);
    L.item = item;
    L.nodes = it->nodes;
    L.woop = it->woop;
    L.node_f4 = it->node_f4;
    L.woop_f4 = it->woop_f4;
    L.out_idx = it->perm ? (int64_t)__ldg(it->perm + local) : local;
    L.gidx = g;
    return it;
}

template <bool MULTI>
__device__ __forceinline__ Ray fetch_ray(const TraceParams& p, int64_t g, Lane& L) {
    // A lane's rays come from a counter that only grows, so its next ray is in
    // its current item or a later one: check the next item's start first, and
    // search only forward when the ray lies beyond it.
    const TraceItem* it = set_lane<MULTI>(p, g, MULTI ? find_item(p, g, L.item) : 0, L);
    const int64_t local = g - (MULTI ? it->ray_begin : 0);
    Ray r;
    r.origin_tmin = __ldcs(&it->rays[local].origin_tmin);
    r.dir_tmax = __ldcs(&it->rays[local].dir_tmax);
    return r;
}

__device__ __forceinline__ void store_hit(Hit* hits, int64_t i, float t, int addr, float u, float v) {
    __stcs(&hits[i].t_triId_u_v, make_float4(t, __int_as_float(addr), u, v));
}

// A finished ray's result: its Hit, or -- for an item with AO counters -- one
// count for its surfel when it is occluded.
template <bool MULTI>
__device__ __forceinline__ void finish_ray(const TraceParams& p, const Lane& L, float t, int addr, float u, float v) {
    const TraceItem* it = MULTI ? p.items + L.item : &p.single;
    uint32_t* counts = it->ao_counts;
    if (counts) {
        if (addr >= 0) atomicAdd(counts + L.out_idx / it->ao_spp, 1u);
    } else {
        store_hit(it->hits, L.out_idx, t, addr, u, v);
    }
}

// ------------------------------------------------------------------ CWBVH --

template <bool ANY, int SMEM, bool MULTI, bool COUNT, bool RING>
__global__ void RQ_KERNEL_BOUNDS cwbvh_kernel(const TraceParams p) {
    extern __shared__ uint2 sstack[];
    constexpr int LOCAL = kStackTotal - SMEM;
    uint2 lstack[LOCAL];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned tid = threadIdx.x;
    const unsigned B = blockDim.x;

    constexpr bool PAIRS = !(MULTI && RING);
    Lane L{};
    float ox = 0.f, oy = 0.f, oz = 0.f, dx = 0.f, dy = 0.f, dz = 0.f, tmin = 0.f, tmax = 0.f;
    float idx_ = 0.f, idy = 0.f, idz = 0.f;
    unsigned octinv = 0, octinv4 = 0;
    uint2 ng = make_uint2(0u, 0u), tg = make_uint2(0u, 0u);
    int sp = 0, hit_addr = -1, steps = 0, nvis = 0, ntri = 0;
    float hu = 0.f, hv = 0.f;
    bool active = false, exhausted = false;
    const float rt = p.postpone_ratio;

    auto push = [&](uint2 v) -> bool {
        if (sp < SMEM) sstack[(unsigned)sp * B + tid] = v;
        else if (sp < kStackTotal) lstack[sp - SMEM] = v;
        else return false;
        ++sp;
        return true;
    };
    auto pop = [&]() -> uint2 {
        --sp;
        return sp < SMEM ? sstack[(unsigned)sp * B + tid] : lstack[sp - SMEM];
    };
    auto finish = [&](unsigned err) {
        if (err) {
            atomicOr(&p.scratch->error, err);
            hit_addr = -1;
        }
        finish_ray<MULTI>(p, L, tmax, hit_addr, hu, hv);
        if (COUNT) {
            p.node_visits[L.gidx] = nvis;
            p.tri_tests[L.gidx] = ntri;
        }
        active = false;
    };

    // Per-warp ray ring after the stacks.
    unsigned char* const ring = reinterpret_cast<unsigned char*>(sstack + (size_t)SMEM * B) +
                                (size_t)(tid >> 5) * kRingBytesPerWarp;
    float4* const ring_ray = reinterpret_cast<float4*>(ring);
    int64_t* const ring_base = reinterpret_cast<int64_t*>(ring + kRingSlots * sizeof(Ray));
    int* const ring_item = reinterpret_cast<int*>(ring + kRingSlots * sizeof(Ray) + 2 * sizeof(int64_t));
    unsigned cons = 0u;  // next slot to hand out (warp-uniform)
    int pf_item = -1;  // item of the lane's last prefetched ray (forward search hint)
    // Takes the next 32 rays from the counter into half `half` of the ring.
    auto claim = [&](unsigned half) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(&p.scratch->ray_counter, (unsigned long long)kRingHalf);
        base = __shfl_sync(kFullMask, base, 0);
        if (lane == 0) ring_base[half] = (int64_t)base;
        const int64_t g = (int64_t)base + lane;
        if (g < p.total_rays) {
            const unsigned slot = half * kRingHalf + lane;
            const int item = MULTI ? find_item(p, g, pf_item) : 0;
            pf_item = item;
            ring_item[slot] = item;
            const TraceItem* it = MULTI ? p.items + item : &p.single;
            const Ray* src = it->rays + (g - (MULTI ? it->ray_begin : 0));
            cp_async16(ring_ray + 2u * slot, &src->origin_tmin);
            cp_async16(ring_ray + 2u * slot + 1u, &src->dir_tmax);
        }
        cp_async_commit();
    };
    if (RING) {
        claim(0u);
        claim(1u);
    }
    auto start = [&](const Ray& r) {
        ox = r.origin_tmin.x; oy = r.origin_tmin.y; oz = r.origin_tmin.z; tmin = r.origin_tmin.w;
        dx = r.dir_tmax.x; dy = r.dir_tmax.y; dz = r.dir_tmax.z; tmax = r.dir_tmax.w;
        idx_ = guarded_rcp(dx);
        idy = guarded_rcp(dy);
        idz = guarded_rcp(dz);
        octinv = 7u - (((dx < 0.f) ? 4u : 0u) | ((dy < 0.f) ? 2u : 0u) | ((dz < 0.f) ? 1u : 0u));
        octinv4 = octinv * 0x01010101u;
        ng = make_uint2(0u, 0x80000000u);
        tg = make_uint2(0u, 0u);
        sp = 0; hit_addr = -1; hu = 0.f; hv = 0.f; steps = 0; nvis = 0; ntri = 0;
        active = true;
    };

    for (;;) {
        // ---- hand rays to idle lanes
        const bool need = !active && !exhausted;
        const unsigned needm = __ballot_sync(kFullMask, need);
        if (RING && needm) {
            // Slots [cons, end) go to the needy lanes in lane order.  The half
            // holding cons was filled before the other one, so its copies are
            // done after waiting for all but the newest group; a refill that
            // runs into the other half waits for that one too.
            const unsigned half_end = (cons & kRingHalf) + kRingHalf;
            const unsigned end = cons + (unsigned)__popc(needm);
            if (end > half_end) cp_async_wait<0>(); else cp_async_wait<1>();
            __syncwarp();
            if (need) {
                const unsigned rank = (unsigned)__popc(needm & lanemask_lt());
                const unsigned slot = (cons + rank) & (kRingSlots - 1u);
                const int64_t g = ring_base[slot / kRingHalf] + (slot & (kRingHalf - 1u));
                if (g < p.total_rays) {
                    set_lane<MULTI>(p, g, MULTI ? ring_item[slot] : 0, L);
                    Ray r;
                    r.origin_tmin = ring_ray[2u * slot];
                    r.dir_tmax = ring_ray[2u * slot + 1u];
                    start(r);
                } else {
                    exhausted = true;
                }
            }
            if (end >= half_end) {  // the half of cons is used up: refill it
                __syncwarp();
                claim((cons / kRingHalf) & 1u);
            }
            cons = end & (kRingSlots - 1u);
        } else if (needm) {
            const int leader = __ffs(needm) - 1;
            unsigned long long base = 0;
            if ((int)lane == leader) base = atomicAdd(&p.scratch->ray_counter, (unsigned long long)__popc(needm));
            base = __shfl_sync(kFullMask, base, leader);
            if (need) {
                const int64_t g = (int64_t)base + __popc(needm & lanemask_lt());
                if (g < p.total_rays) {
                    start(fetch_ray<MULTI>(p, g, L));
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(kFullMask, active) == 0u) break;

        int lost = 0;
        for (;;) {
            // ---- node phase: take the nearest child of the current node group
            auto node_step = [&]() -> unsigned {
                unsigned fault = 0u;
                const unsigned hitsm = ng.y;
                const unsigned bit = highest_bit(hitsm);
                const unsigned base = ng.x;
                ng.y &= ~(1u << bit);
                if (ng.y > 0x00FFFFFFu && !push(ng)) fault = kErrStackOverflow;
                const unsigned slot = (bit - 24u) ^ octinv;
                const unsigned ci = base + (unsigned)__popc(hitsm & ~(0xFFFFFFFFu << slot));
                if (++steps > p.step_limit) fault |= kErrTimeout;
                if ((uint64_t)ci * 5u + 5u > (uint64_t)L.node_f4) fault |= kErrBadScene;
                if (!fault) {
                    const float4* np = L.nodes + (size_t)ci * 5u;
                    const float4 n0 = ld_nc(np + 0), n1 = ld_nc(np + 1), n2 = ld_nc(np + 2);
                    const float4 n3 = ld_nc(np + 3), n4 = ld_nc(np + 4);
                    if (COUNT) ++nvis;
                    const unsigned ew = __float_as_uint(n0.w);
                    const float adjx = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)(ew & 0xFFu) + 127)) << 23), idx_);
                    const float adjy = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)((ew >> 8) & 0xFFu) + 127)) << 23), idy);
                    const float adjz = __fmul_rn(__uint_as_float(((unsigned)((int)(signed char)((ew >> 16) & 0xFFu) + 127)) << 23), idz);
                    const float orx = __fmul_rn(-__fsub_rn(ox, n0.x), idx_);
                    const float ory = __fmul_rn(-__fsub_rn(oy, n0.y), idy);
                    const float orz = __fmul_rn(-__fsub_rn(oz, n0.z), idz);
                    const bool negx = idx_ < 0.f, negy = idy < 0.f, negz = idz < 0.f;
                    const unsigned hitmask = cwbvh_hitmask(n1, n2, n3, n4, adjx, adjy, adjz, orx, ory, orz, negx,
                                                           negy, negz, octinv4, tmin, tmax);
                    ng = make_uint2(__float_as_uint(n1.x), (hitmask & 0xFF000000u) | (ew >> 24));
                    tg = make_uint2(__float_as_uint(n1.y), hitmask & 0x00FFFFFFu);
                }
                return fault;
            };
            unsigned fault = 0u;
            if (active) {
                if (ng.y > 0x00FFFFFFu) {
                    fault = node_step();
                } else {
                    tg = ng;
                    ng = make_uint2(0u, 0u);
                }
                if (fault) finish(fault);
            }
            // Any-hit: a lane whose node produced no triangles and has inner
            // children left descends once more in the same iteration, in the
            // order the next iteration would take (+2 % batched any-hit;
            // closest-hit loses 6-10 %: its triangle tests, which shrink
            // tmax, get postponed more often).
            if (ANY && __ballot_sync(kFullMask, active && tg.y == 0u && ng.y > 0x00FFFFFFu)) {
                if (active && tg.y == 0u && ng.y > 0x00FFFFFFu) {
                    const unsigned f2 = node_step();
                    if (f2) finish(f2);
                }
            }

            // ---- triangle phase, warp-synchronous; postpone when few lanes remain
            {
                const int total = __popc(__ballot_sync(kFullMask, active));
                const int threshold = (int)((float)total * rt);
                for (;;) {
                    const bool want = active && tg.y != 0u;
                    const unsigned wm = __ballot_sync(kFullMask, want);
                    if (wm == 0u) break;
                    if (__popc(wm) < threshold) {
                        if (want && !push(tg)) finish(kErrStackOverflow);
                        break;
                    }
                    if (want) {
                        // Two triangles of the lane's group per round when it
                        // has two (PAIRS), in the group's order: the second is
                        // tested against the tmax the first left, and not at
                        // all once an any-hit ray has finished (fewer
                        // warp-wide votes per triangle: +1.0-2.2 % on single
                        // scenes, +1.3 % on the 64-scene closest-hit batch,
                        // +2.0 % on a one-item batch; the ring batch kernel
                        // measured 0.5-1.1 % slower with it on the 64-scene
                        // AO batch and tests one per round).
                        const unsigned ti = highest_bit(tg.y);
                        const unsigned tri = tg.x * 3u + ti * 3u;
                        tg.y &= ~(1u << ti);
                        const bool two = PAIRS && tg.y != 0u;
                        unsigned tri2 = tri;
                        if (two) {
                            const unsigned ti2 = highest_bit(tg.y);
                            tri2 = tg.x * 3u + ti2 * 3u;
                            tg.y &= ~(1u << ti2);
                        }
                        if ((uint64_t)tri + 3u > (uint64_t)L.woop_f4) {
                            finish(kErrBadScene);
                        } else {
                            const float4* tp = L.woop + tri;
                            if (COUNT) ++ntri;
                            float t, u, v;
                            const float4 v0 = ld_nc(tp), v1 = ld_nc(tp + 1), v2 = ld_nc(tp + 2);
                            if (woop_test(v0, v1, v2, ox, oy, oz, dx, dy, dz, tmin, tmax, t, u, v)) {
                                tmax = t;
                                hit_addr = (int)tri;
                                hu = u;
                                hv = v;
                                if (ANY) finish(0u);
                            }
                            if (two && active) {
                                if ((uint64_t)tri2 + 3u > (uint64_t)L.woop_f4) {
                                    finish(kErrBadScene);
                                } else {
                                    const float4* tp2 = L.woop + tri2;
                                    if (COUNT) ++ntri;
                                    const float4 w0 = ld_nc(tp2), w1 = ld_nc(tp2 + 1), w2 = ld_nc(tp2 + 2);
                                    if (woop_test(w0, w1, w2, ox, oy, oz, dx, dy, dz, tmin, tmax, t, u, v)) {
                                        tmax = t;
                                        hit_addr = (int)tri2;
                                        hu = u;
                                        hv = v;
                                        if (ANY) finish(0u);
                                    }
                                }
                            }
                        }
                    }
                }
            }

            // ---- continue with the stack, or finish the ray
            if (active && ng.y <= 0x00FFFFFFu) {
                if (sp > 0) ng = pop();
                else finish(0u);
            }

            const unsigned am = __ballot_sync(kFullMask, active);
            if (am == 0u) break;
            lost += 32 - __popc(am) - p.fetch_nd;
            if (lost >= p.fetch_nw) break;
        }
    }
    if (RING) cp_async_wait<0>();  // no copy into the ring outlives the block
}

// ------------------------------------------------------------------- BVH2 --

template <bool ANY, int SMEM, bool MULTI, bool COUNT>
__global__ void RQ_BVH2_BOUNDS bvh2_kernel(const TraceParams p) {
    extern __shared__ int istack[];
    constexpr int LOCAL = kStackTotal - SMEM;
    int lstack[LOCAL];
    const unsigned lane = threadIdx.x & 31u;
    const unsigned tid = threadIdx.x;
    const unsigned B = blockDim.x;
    const bool speculate = p.bvh2_speculative != 0;

    Lane L{};
    float ox = 0.f, oy = 0.f, oz = 0.f, dx = 0.f, dy = 0.f, dz = 0.f, tmin = 0.f, tmax = 0.f;
    float idx_ = 0.f, idy = 0.f, idz = 0.f, oodx = 0.f, oody = 0.f, oodz = 0.f;
    int node = 0, leaf = 0, tcur = 0, sp = 0, hit_addr = -1, steps = 0, nvis = 0, ntri = 0;
    float hu = 0.f, hv = 0.f;
    bool active = false, exhausted = false;

    // Stack slot 0 holds the sentinel; entries 1.. are pushed far children.
    auto push = [&](int v) -> bool {
        ++sp;
        if (sp < SMEM) istack[(unsigned)sp * B + tid] = v;
        else if (sp < kStackTotal) lstack[sp - SMEM] = v;
        else { --sp; return false; }
        return true;
    };
    auto pop = [&]() -> int {
        const int v = sp == 0 ? (int)kBvh2Sentinel : (sp < SMEM ? istack[(unsigned)sp * B + tid] : lstack[sp - SMEM]);
        if (sp > 0) --sp;
        return v;
    };
    auto finish = [&](unsigned err) {
        if (err) {
            atomicOr(&p.scratch->error, err);
            hit_addr = -1;
        }
        finish_ray<MULTI>(p, L, tmax, hit_addr, hu, hv);
        if (COUNT) {
            p.node_visits[L.gidx] = nvis;
            p.tri_tests[L.gidx] = ntri;
        }
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
                    const Ray r = fetch_ray<MULTI>(p, g, L);
                    ox = r.origin_tmin.x; oy = r.origin_tmin.y; oz = r.origin_tmin.z; tmin = r.origin_tmin.w;
                    dx = r.dir_tmax.x; dy = r.dir_tmax.y; dz = r.dir_tmax.z; tmax = r.dir_tmax.w;
                    idx_ = guarded_rcp(dx);
                    idy = guarded_rcp(dy);
                    idz = guarded_rcp(dz);
                    oodx = __fmul_rn(ox, idx_);
                    oody = __fmul_rn(oy, idy);
                    oodz = __fmul_rn(oz, idz);
                    node = 0; leaf = 0; sp = 0; hit_addr = -1; hu = 0.f; hv = 0.f; steps = 0; nvis = 0; ntri = 0;
                    active = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (__ballot_sync(kFullMask, active) == 0u) break;

        int lost = 0;
        for (;;) {
            // ---- inner-node loop (src/TraversalKernelBVH2.cu:70-122)
            if (active) leaf = 0;
            for (;;) {
                const bool in = active && node != (int)kBvh2Sentinel && node >= 0 && (speculate || leaf >= 0);
                if (__ballot_sync(kFullMask, in) == 0u) break;
                if (in) {
                    unsigned fault = 0u;
                    if (++steps > p.step_limit) fault |= kErrTimeout;
                    if ((uint64_t)(unsigned)node + 4u > (uint64_t)L.node_f4) fault |= kErrBadScene;
                    if (!fault) {
                        const float4* np = L.nodes + node;
                        const float4 n0 = ld_nc(np), n1 = ld_nc(np + 1), n2 = ld_nc(np + 2), n3 = ld_nc(np + 3);
                        if (COUNT) ++nvis;
                        // Slabs: lo * idir - ood (src/TraversalKernelBVH2.cu:16-19).
                        const float a0lx = __fmaf_rn(n0.x, idx_, -oodx), a0hx = __fmaf_rn(n0.y, idx_, -oodx);
                        const float a0ly = __fmaf_rn(n0.z, idy, -oody), a0hy = __fmaf_rn(n0.w, idy, -oody);
                        const float a0lz = __fmaf_rn(n2.x, idz, -oodz), a0hz = __fmaf_rn(n2.y, idz, -oodz);
                        const float a1lx = __fmaf_rn(n1.x, idx_, -oodx), a1hx = __fmaf_rn(n1.y, idx_, -oodx);
                        const float a1ly = __fmaf_rn(n1.z, idy, -oody), a1hy = __fmaf_rn(n1.w, idy, -oody);
                        const float a1lz = __fmaf_rn(n2.z, idz, -oodz), a1hz = __fmaf_rn(n2.w, idz, -oodz);
                        const float c0min = imin_then_max(a0lz, a0hz, imin_then_max(a0ly, a0hy, imin_then_max(a0lx, a0hx, tmin)));
                        const float c0max = imax_then_min(a0lz, a0hz, imax_then_min(a0ly, a0hy, imax_then_min(a0lx, a0hx, tmax)));
                        const float c1min = imin_then_max(a1lz, a1hz, imin_then_max(a1ly, a1hy, imin_then_max(a1lx, a1hx, tmin)));
                        const float c1max = imax_then_min(a1lz, a1hz, imax_then_min(a1ly, a1hy, imax_then_min(a1lx, a1hx, tmax)));
                        const bool t0 = c0min <= c0max, t1 = c1min <= c1max;
                        int cx = __float_as_int(n3.x), cy = __float_as_int(n3.y);
                        if (!t0 && !t1) {
                            node = pop();
                        } else {
                            node = t0 ? cx : cy;
                            if (t0 && t1) {
                                if (c1min < c0min) { const int tmp = node; node = cy; cy = tmp; }
                                if (!push(cy)) fault |= kErrStackOverflow;
                            }
                        }
                        if (!fault && node < 0 && leaf >= 0) {
                            leaf = node;
                            node = pop();
                        }
                    }
                    if (fault) finish(fault);
                }
                if (speculate && __ballot_sync(kFullMask, in && leaf >= 0) == 0u) break;
            }

            // ---- leaf loop, one triangle per iteration (src/TraversalKernelBVH2.cu:124-169)
            if (active && leaf < 0) tcur = ~leaf;
            for (;;) {
                const bool want = active && leaf < 0;
                if (__ballot_sync(kFullMask, want) == 0u) break;
                if (want) {
                    if ((uint64_t)(unsigned)tcur + 1u > (uint64_t)L.woop_f4) {
                        finish(kErrBadScene);
                    } else {
                        const float4 v0 = ld_nc(L.woop + tcur);
                        if (__float_as_uint(v0.x) == 0x80000000u) {
                            // Leaf terminator: move to the postponed node / next leaf.
                            leaf = node;
                            if (node < 0) {
                                node = pop();
                                tcur = ~leaf;
                            }
                        } else if ((uint64_t)(unsigned)tcur + 3u > (uint64_t)L.woop_f4) {
                            finish(kErrBadScene);
                        } else {
                            const float4 v1 = ld_nc(L.woop + tcur + 1), v2 = ld_nc(L.woop + tcur + 2);
                            if (COUNT) ++ntri;
                            float t, u, v;
                            if (woop_test(v0, v1, v2, ox, oy, oz, dx, dy, dz, tmin, tmax, t, u, v)) {
                                tmax = t;
                                hit_addr = tcur;
                                hu = u;
                                hv = v;
                                if (ANY) finish(0u);
                            }
                            tcur += 3;
                        }
                    }
                }
            }

            if (active && node == (int)kBvh2Sentinel) finish(0u);

            const unsigned am = __ballot_sync(kFullMask, active);
            if (am == 0u) break;
            lost += 32 - __popc(am) - p.fetch_nd;
            if (lost >= p.fetch_nw) break;
        }
    }
}

// ---------------------------------------------------------------- launch --

template <bool MULTI, bool COUNT, bool RING>
static TraceKernelFn select_cwbvh(bool any, int smem) {
#define RQ_CW(A, S) (TraceKernelFn)cwbvh_kernel<A, S, MULTI, COUNT, RING>
    if (any) return smem <= 4 ? RQ_CW(true, 4) : (smem <= 8 ? RQ_CW(true, 8) : RQ_CW(true, 16));
    return smem <= 4 ? RQ_CW(false, 4) : (smem <= 8 ? RQ_CW(false, 8) : RQ_CW(false, 16));
#undef RQ_CW
}
template <bool MULTI, bool COUNT>
static TraceKernelFn select_bvh2(bool any, int smem) {
#define RQ_B2(A, S) (TraceKernelFn)bvh2_kernel<A, S, MULTI, COUNT>
    if (any) return smem <= 4 ? RQ_B2(true, 4) : (smem <= 8 ? RQ_B2(true, 8) : RQ_B2(true, 16));
    return smem <= 4 ? RQ_B2(false, 4) : (smem <= 8 ? RQ_B2(false, 8) : RQ_B2(false, 16));
#undef RQ_B2
}

TraceKernelFn trace_kernel(rq_bvh_kind kind, bool any, int smem, bool multi, bool count, bool ring) {
    if (kind == RQ_BVH_CWBVH) {
        if (count) return select_cwbvh<false, true, false>(any, smem);
        if (ring && any) {  // any-hit only (closest-hit batches measured 1 % slower with the ring)
            if (multi)
                return smem <= 4 ? (TraceKernelFn)cwbvh_kernel<true, 4, true, false, true>
                                 : (smem <= 8 ? (TraceKernelFn)cwbvh_kernel<true, 8, true, false, true>
                                              : (TraceKernelFn)cwbvh_kernel<true, 16, true, false, true>);
            return smem <= 4 ? (TraceKernelFn)cwbvh_kernel<true, 4, false, false, true>
                             : (smem <= 8 ? (TraceKernelFn)cwbvh_kernel<true, 8, false, false, true>
                                          : (TraceKernelFn)cwbvh_kernel<true, 16, false, false, true>);
        }
        if (!multi) return select_cwbvh<false, false, false>(any, smem);
        return select_cwbvh<true, false, false>(any, smem);
    }
    if (count) return select_bvh2<false, true>(any, smem);
    return multi ? select_bvh2<true, false>(any, smem) : select_bvh2<false, false>(any, smem);
}

int smem_entries_of(int requested) { return requested <= 4 ? 4 : (requested <= 8 ? 8 : 16); }

size_t trace_smem_bytes(rq_bvh_kind kind, int smem_entries, int block, bool ring) {
    if (kind != RQ_BVH_CWBVH) return sizeof(int) * (size_t)smem_entries * (size_t)block;
    return sizeof(uint2) * (size_t)smem_entries * (size_t)block +
           (ring ? kRingBytesPerWarp * (size_t)(block / 32) : 0);
}

}  // namespace rq
