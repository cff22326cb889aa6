// Bandwidth probe used by the benchmark for the L2 roofline of the traversal
// kernels: the scenes of the small and batched workloads are L2-resident, so
// their node and triangle fetches are bounded by L2, not HBM, bandwidth.
//
// Access pattern: a warp's load instruction covers 512 contiguous bytes (32
// lanes x 16 B), so every 32-byte L2 sector it requests is used whole; each
// thread keeps LOADS such loads in flight, one grid stride apart.
#include <cuda_runtime.h>
#include <stdint.h>

#include "runtime.h"

namespace rq {

template <int LOADS>
__global__ void __launch_bounds__(256) l2_read_kernel(const uint4* __restrict__ buf, int64_t n16, int reps,
                                                      uint32_t* __restrict__ sink) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (int r = 0; r < reps; ++r) {
        for (int64_t i = first; i < n16; i += LOADS * stride) {
            uint4 v[LOADS];
#pragma unroll
            for (int k = 0; k < LOADS; ++k) {
                const int64_t j = i + k * stride;
                v[k] = j < n16 ? __ldcg(buf + j) : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int k = 0; k < LOADS; ++k) acc ^= v[k].x ^ v[k].y ^ v[k].z ^ v[k].w;
        }
        acc = (acc << 1) | (acc >> 31);
    }
    if (acc == 0x9E3779B9u) *sink = acc;
}

rq_status probe_l2(const void* buf, int64_t bytes, int reps, int blocks_per_sm, int loads, uint32_t* sink,
                   void* stream) {
    if (!buf || !sink || bytes <= 0 || (bytes % 16) != 0 || reps <= 0 || ((uintptr_t)buf % 16) != 0 ||
        blocks_per_sm <= 0 || blocks_per_sm > 64 || (loads != 4 && loads != 8))
        return RQ_ERR_INVALID_ARG;
    int dev = 0;
    RQ_CUDA(cudaGetDevice(&dev));
    int sms = 0;
    RQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const dim3 grid((unsigned)(sms * blocks_per_sm));
    if (loads == 4)
        l2_read_kernel<4><<<grid, 256, 0, (cudaStream_t)stream>>>((const uint4*)buf, bytes / 16, reps, sink);
    else
        l2_read_kernel<8><<<grid, 256, 0, (cudaStream_t)stream>>>((const uint4*)buf, bytes / 16, reps, sink);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

}  // namespace rq

using namespace rq;

extern "C" rq_status rq_probe_l2_read(const void* buf, int64_t bytes, int reps, uint32_t* sink, void* stream) {
    return probe_l2(buf, bytes, reps, 8, 4, sink, stream);
}

extern "C" rq_status rq_probe_l2_read_shape(const void* buf, int64_t bytes, int reps, int blocks_per_sm, int loads,
                                           uint32_t* sink, void* stream) {
    return probe_l2(buf, bytes, reps, blocks_per_sm, loads, sink, stream);
}
