// Bandwidth probe used by the benchmark for the L2 roofline of the traversal
// kernels: the scenes of the small and batched workloads are L2-resident, so
// their node and triangle fetches are bounded by L2, not HBM, bandwidth.
#include <cuda_runtime.h>
#include <stdint.h>

#include "runtime.h"

namespace rq {

// Four independent 16-byte L2 loads in flight per thread per iteration.
__global__ void __launch_bounds__(256) l2_read_kernel(const uint4* __restrict__ buf, int64_t n64, int reps,
                                                      uint32_t* __restrict__ sink) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t acc = 0;
    for (int r = 0; r < reps; ++r) {
        for (int64_t i = first; i < n64; i += stride) {
            const uint4* q = buf + 4 * i;
            const uint4 a = __ldcg(q), b = __ldcg(q + 1), c = __ldcg(q + 2), d = __ldcg(q + 3);
            acc ^= a.x ^ a.y ^ a.z ^ a.w ^ b.x ^ b.y ^ b.z ^ b.w ^ c.x ^ c.y ^ c.z ^ c.w ^ d.x ^ d.y ^ d.z ^ d.w;
        }
        acc = (acc << 1) | (acc >> 31);
    }
    if (acc == 0x9E3779B9u) *sink = acc;
}

}  // namespace rq

using namespace rq;

extern "C" rq_status rq_probe_l2_read(const void* buf, int64_t bytes, int reps, uint32_t* sink, void* stream) {
    if (!buf || !sink || bytes <= 0 || (bytes % 64) != 0 || reps <= 0 || ((uintptr_t)buf % 16) != 0)
        return RQ_ERR_INVALID_ARG;
    int dev = 0;
    RQ_CUDA(cudaGetDevice(&dev));
    int sms = 0;
    RQ_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    l2_read_kernel<<<sms * 8, 256, 0, (cudaStream_t)stream>>>((const uint4*)buf, bytes / 64, reps, sink);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}
