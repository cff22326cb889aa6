// rq_sort_rays_static: the Morton ray sort of rq_sort_rays without any
// device allocation.
//
// Some callers cannot call cudaMalloc: a plugin running inside a host
// application that owns all device memory through its own pool, or a service
// whose device-memory budget was fixed when it started.  rq_sort_rays creates
// its sort buffers on every call, so such callers use this entry point
// instead.  Its scratch (keys, values, the one-item table and the radix-sort
// temp storage) lives in one file-scope device array of kScratchBytes, which
// every GPU that loads librq holds until the process exits; that bounds a
// call to RQ_SORT_STATIC_MAX_RAYS rays.
//
// The pipeline is rq_sort_rays's own: the same key and gather kernels and the
// same radix sort, so the outputs are identical.  The one-item table and the
// bounds are written into the array by a one-thread kernel that receives them
// as launch arguments, so no host memory is read after the call returns.
//
// Set-up: the first call on each device (with that device current) looks up
// the array's device address with cudaGetSymbolAddress and sizes the sort's
// temp storage; make that first call before any stream capture.  Every call
// shares the array and leaves its contents behind; each call writes every
// scratch byte it reads, so nothing needs clearing.  Calls whose work
// overlaps on the GPU (other streams, other host threads) race on the array.
// The call is stream-ordered: it returns with its work queued on `stream`.
#include <cub/device/device_radix_sort.cuh>

#include <mutex>
#include <string>

#include "runtime.h"

namespace rq {

// Defined in rays.cu (the kernels rq_sort_rays launches).
__global__ void morton_keys_kernel(const TraceItem* __restrict__ items, int n_items, const float* __restrict__ bounds,
                                   int64_t total, uint64_t* __restrict__ keys, int32_t* __restrict__ vals);
__global__ void gather_rays_kernel(const TraceItem* __restrict__ items, const uint64_t* __restrict__ keys,
                                   const int32_t* __restrict__ vals, int64_t total, Ray* __restrict__ sorted);

namespace {

// Writes the one-item table and the bounds into the static scratch.
__global__ void static_sort_setup_kernel(TraceItem item, float3 lo, float3 hi, TraceItem* items, float* bounds) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        items[0] = item;
        bounds[0] = lo.x; bounds[1] = lo.y; bounds[2] = lo.z;
        bounds[3] = hi.x; bounds[4] = hi.y; bounds[5] = hi.z;
    }
}

constexpr int64_t kMaxRays = RQ_SORT_STATIC_MAX_RAYS;
constexpr size_t kScratchBytes = 20u << 20;  // 20 MiB: 10 MiB of keys/values + the sort's ~6.1 MiB temp
constexpr int kEndBit = 33;                   // one item: 32 key bits + 1 item bit, as rq_sort_rays uses

static __device__ __align__(256) unsigned char g_sort_scratch[kScratchBytes];

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets inside the array.
constexpr size_t kItemOff = 0;
constexpr size_t kBoundsOff = align256(kItemOff + sizeof(TraceItem));
constexpr size_t kKeysInOff = align256(kBoundsOff + 6 * sizeof(float));
constexpr size_t kKeysOutOff = align256(kKeysInOff + sizeof(uint64_t) * kMaxRays);
constexpr size_t kValsInOff = align256(kKeysOutOff + sizeof(uint64_t) * kMaxRays);
constexpr size_t kTempOff = align256(kValsInOff + sizeof(int32_t) * kMaxRays);
static_assert(kTempOff < kScratchBytes, "static sort scratch too small for its fixed buffers");

struct DeviceState {
    bool ready = false;
    rq_status status = RQ_OK;
    unsigned char* base = nullptr;  // device address of g_sort_scratch on this device
    size_t temp_bytes = 0;          // radix-sort temp storage for kMaxRays
};

std::mutex g_mu;
constexpr int kMaxDevices = 64;
DeviceState g_state[kMaxDevices];

rq_status setup(int dev, DeviceState** out) {
    if (dev < 0 || dev >= kMaxDevices) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceState& s = g_state[dev];
    if (!s.ready) {
        s.ready = true;
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess) {
            s.status = cuda_fail(e, "rq_sort_rays_static: cudaGetSymbolAddress");
        } else {
            s.base = static_cast<unsigned char*>(p);
            size_t bytes = 0;
            e = cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const uint64_t*)nullptr, (uint64_t*)nullptr,
                                                (const int32_t*)nullptr, (int32_t*)nullptr, kMaxRays, 0, kEndBit);
            if (e != cudaSuccess) {
                s.status = cuda_fail(e, "rq_sort_rays_static: sizing the radix sort");
            } else if (kTempOff + bytes > kScratchBytes) {
                set_last_error("rq_sort_rays_static: the radix sort needs " + std::to_string(bytes) +
                               " bytes of temp storage, more than the static scratch holds");
                s.status = RQ_ERR_OOM;
            } else {
                s.temp_bytes = bytes;
            }
        }
    }
    *out = &s;
    return s.status;
}

unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

}  // namespace
}  // namespace rq

using namespace rq;

extern "C" rq_status rq_sort_rays_static(const rq_ray* rays, int64_t count, const float bounds_lo[3],
                                         const float bounds_hi[3], rq_ray* sorted_rays, int32_t* perm,
                                         void* stream) {
    if (count < 0 || (count > 0 && (!rays || !sorted_rays || !perm || !bounds_lo || !bounds_hi)))
        return RQ_ERR_INVALID_ARG;
    if (count > kMaxRays) {
        set_last_error("rq_sort_rays_static: " + std::to_string(count) + " rays exceed its static scratch limit of " +
                       std::to_string(kMaxRays) + " rays; use rq_sort_rays");
        return RQ_ERR_INVALID_ARG;
    }
    if (count == 0) return RQ_OK;
    int dev = 0;
    RQ_CUDA(cudaGetDevice(&dev));
    DeviceState* s = nullptr;
    const rq_status st = setup(dev, &s);
    if (st != RQ_OK) return st;

    cudaStream_t strm = (cudaStream_t)stream;
    unsigned char* b = s->base;
    TraceItem item{};
    item.rays = reinterpret_cast<const Ray*>(rays);
    item.ray_begin = 0;
    item.count = count;
    auto* items = reinterpret_cast<TraceItem*>(b + kItemOff);
    auto* bounds = reinterpret_cast<float*>(b + kBoundsOff);
    static_sort_setup_kernel<<<1, 32, 0, strm>>>(item, make_float3(bounds_lo[0], bounds_lo[1], bounds_lo[2]),
                                                  make_float3(bounds_hi[0], bounds_hi[1], bounds_hi[2]), items,
                                                  bounds);
    RQ_CUDA(cudaGetLastError());
    auto* keys_in = reinterpret_cast<uint64_t*>(b + kKeysInOff);
    auto* keys_out = reinterpret_cast<uint64_t*>(b + kKeysOutOff);
    auto* vals_in = reinterpret_cast<int32_t*>(b + kValsInOff);
    morton_keys_kernel<<<blocks_for(count, 256), 256, 0, strm>>>(items, 1, bounds, count, keys_in, vals_in);
    RQ_CUDA(cudaGetLastError());
    size_t tb = s->temp_bytes;
    RQ_CUDA(cub::DeviceRadixSort::SortPairs(b + kTempOff, tb, keys_in, keys_out, vals_in, perm, count, 0, kEndBit,
                                            strm));
    gather_rays_kernel<<<blocks_for(count, 256), 256, 0, strm>>>(items, keys_out, perm, count,
                                                                 reinterpret_cast<Ray*>(sorted_rays));
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}
