// Internal interface between librq's host runtime and its CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rq.h"

namespace rq {

// Byte-identical to the reference's Ray / Hit (src/helper_math.h:1853-1865).
struct Ray {
    float4 origin_tmin;
    float4 dir_tmax;
};
struct Hit {
    float4 t_triId_u_v;
};
static_assert(sizeof(Ray) == 32 && sizeof(Hit) == 16, "Ray/Hit layout");
static_assert(sizeof(rq_ray) == 32 && sizeof(rq_hit) == 16, "rq_ray/rq_hit layout");

// Error bits a kernel may set in its context's error word.
enum : unsigned {
    kErrStackOverflow = 1u,
    kErrTimeout = 2u,
    kErrBadScene = 4u,
};

// Device scratch of one context: the dynamic-fetch counter and the error word.
constexpr int kDefaultStepLimit = 1 << 22;  // node visits per ray before kErrTimeout (rq_launch.step_limit = 0)

struct DevScratch {
    unsigned long long ray_counter;
    unsigned int error;
    unsigned int pad;
};

// One (scene, rays, hits) unit of work.  Rays [0, count) of this item are the
// global rays [ray_begin, ray_begin + count).  With perm set, ray k is written
// to hits[perm[k]] (the rays were reordered before tracing).
struct TraceItem {
    const float4* nodes;
    const float4* woop;
    const Ray* rays;
    Hit* hits;
    const int32_t* perm;
    int64_t ray_begin;
    int64_t count;
    uint32_t node_f4;  // node buffer length in float4 (bounds checks)
    uint32_t woop_f4;  // Woop buffer length in float4
    uint32_t* ao_counts;  // non-null: occluded rays are counted per surfel here instead of writing hits
    int32_t ao_spp;       // rays per surfel (consecutive) when ao_counts is set
    int32_t pad;
};

struct TraceParams {
    TraceItem single;         // the scene when the kernel is not a batch kernel
    const TraceItem* items;   // device array of n_items (batch kernels)
    int n_items;
    int64_t total_rays;
    DevScratch* scratch;
    int32_t* node_visits;     // per global ray, counting kernels only
    int32_t* tri_tests;
    float postpone_ratio;
    int fetch_nd;
    int fetch_nw;
    int bvh2_speculative;
    int step_limit;           // node visits per ray before kErrTimeout
};

typedef void (*TraceKernelFn)(TraceParams);

// ring: the CWBVH any-hit kernel that prefetches rays into a per-warp ring
// in shared memory (see trace.cu), for batches of at least
// kRingMinRaysPerThread rays per thread of the grid and single-scene launches
// of at least kRingMinRaysPerThreadSingle (which have no item search to hide).
constexpr int64_t kRingMinRaysPerThread = 64;
constexpr int64_t kRingMinRaysPerThreadSingle = 256;
TraceKernelFn trace_kernel(rq_bvh_kind kind, bool any, int smem, bool multi, bool count, bool ring);
int smem_entries_of(int requested);
size_t trace_smem_bytes(rq_bvh_kind kind, int smem_entries, int block, bool ring);

}  // namespace rq
