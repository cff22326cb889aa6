// Internal runtime objects behind the C ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "device_api.h"

struct rq_ctx {
    int device = 0;
    rq::DevScratch* scratch = nullptr;  // device
    void* temp = nullptr;               // grow-on-demand device temp (sorting)
    size_t temp_bytes = 0;
};

struct rq_scene {
    rq_bvh_kind kind;
    int device = 0;
    const float4* nodes = nullptr;
    const float4* woop = nullptr;
    const int32_t* prim_index = nullptr;
    int64_t node_f4 = 0, woop_f4 = 0, prim_count = 0;
    bool owned = false;
    float lo[3] = {0.f, 0.f, 0.f};
    float hi[3] = {0.f, 0.f, 0.f};
};

namespace rq {

// Records a failing CUDA call for rq_last_error and maps it to a status.
rq_status cuda_fail(cudaError_t e, const char* what);
// Sets the text rq_last_error returns on this thread.
void set_last_error(const std::string& msg);

#define RQ_CUDA(call)                                          \
    do {                                                       \
        cudaError_t rq_e_ = (call);                            \
        if (rq_e_ != cudaSuccess) return rq::cuda_fail(rq_e_, #call); \
    } while (0)

int device_sms(int device);

// Fills zero fields of `l` with defaults for this BVH kind / query.
rq_launch resolve_launch(rq_bvh_kind kind, rq_query q, const rq_launch* l);

// Persistent-grid launch of a trace kernel variant.
rq_status launch_trace(rq_bvh_kind kind, rq_query q, const rq_launch& l, bool multi, bool count,
                       const TraceParams& p, cudaStream_t s);

// Computes the occupancy of a kernel variant ahead of a stream capture.
void warm_launch_cache(rq_bvh_kind kind, rq_query q, const rq_launch& l, bool multi, bool count);

// Zeroes the context's ray counter on the stream.
rq_status reset_counter(rq_ctx* ctx, cudaStream_t s);

TraceItem scene_item(const rq_scene* sc, const rq_ray* rays, rq_hit* hits, int64_t count);
TraceParams base_params(rq_ctx* ctx, const rq_launch& l);

// AO rays of n_surfels surfels (rays.cu); ray k of the call is ray
// first_ray + k of the request it belongs to (its random stream).
rq_status aorays_launch(const float* pos, const float* nrm, const float* radius, int64_t n_surfels, int spp,
                        int64_t first_ray, uint64_t seed, float tmin, float tmax, float offset_scale, rq_ray* out_rays,
                        void* stream);

// Morton keys + radix sort of the rays of several items (rays.cu).
struct SortPlan {
    int n_items = 0;
    int64_t total = 0;
    // device arrays
    uint64_t* keys_in = nullptr;
    uint64_t* keys_out = nullptr;
    int32_t* vals_in = nullptr;
    int32_t* vals_out = nullptr;
    Ray* sorted = nullptr;
    TraceItem* src_items = nullptr;  // items with original rays, ray_begin = offset in sorted order
    float* bounds = nullptr;         // 6 floats per item
    void* cub_temp = nullptr;
    size_t cub_temp_bytes = 0;
    int end_bit = 64;
    int n_kernels = 0;  // kernels one sort_plan_run launches (counted from a captured graph)
};
rq_status sort_plan_create(const std::vector<TraceItem>& items, const std::vector<float>& bounds, SortPlan& plan);
rq_status sort_plan_run(SortPlan& plan, cudaStream_t s);
void sort_plan_destroy(SortPlan& plan);
int sort_plan_kernel_count(const SortPlan& plan);

}  // namespace rq
