// One ray buffer traced over several GPUs that hold replicas of one scene.
//
// Rays are independent, so the work splits into contiguous ray ranges, one
// per device, with no exchange between devices while they trace.  The
// caller's rays and hits live on the home device (the first one).  Range 0 is
// traced there in place; every other device copies its range from the home
// device into its own staging buffer (a peer copy over NVLink, landing in
// local memory), traces it with its own context and stream, and copies its
// hits back into the caller's hit buffer.  This is the multi-GPU form of the
// reference's one-scene entry point rtTraceCWBVH / rtTraceBVH2
// (src/TraversalKernelCWBVH.cu:387-426, src/TraversalKernelBVH2.cu:190-227):
// synchronous like them, with the same Ray / Hit layouts.
//
// No kernel waits on another device: each device's work is ordered on its own
// stream and the host waits for all of them at the end.
#include <algorithm>
#include <vector>

#include "runtime.h"

struct rq_sharded {
    struct Part {
        int device = 0;
        rq_scene_t scene = nullptr;
        rq_ctx_t ctx = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t ready = nullptr;  // recorded on the home stream: the caller's rays are in place
        rq_ray* rays = nullptr;       // staging (not for part 0)
        rq_hit* hits = nullptr;
    };
    std::vector<Part> parts;
    int64_t max_rays = 0;
    int64_t capacity = 0;  // rays per staging buffer
};

namespace {

using rq::cuda_fail;

// Makes `dev` current for the lifetime of the guard, then restores the
// caller's device.
struct DeviceGuard {
    int prev = -1;
    cudaError_t err = cudaSuccess;
    explicit DeviceGuard(int dev) {
        err = cudaGetDevice(&prev);
        if (err == cudaSuccess) err = cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

void destroy_parts(rq_sharded* s) {
    for (auto& p : s->parts) {
        DeviceGuard g(p.device);
        if (p.rays) cudaFree(p.rays);
        if (p.hits) cudaFree(p.hits);
        if (p.ready) cudaEventDestroy(p.ready);
        if (p.stream) cudaStreamDestroy(p.stream);
        if (p.ctx) rq_ctx_destroy(p.ctx);
    }
    s->parts.clear();
}

}  // namespace

namespace rq {

// Range k of `count` rays over n parts: sizes differ by at most one, the
// larger ranges first.
void shard_range(int64_t count, int n, int k, int64_t* begin, int64_t* size) {
    const int64_t q = count / n, r = count % n;
    *begin = k * q + std::min<int64_t>(k, r);
    *size = q + (k < r ? 1 : 0);
}

}  // namespace rq

extern "C" {

rq_status rq_shard_range(int64_t count, int n_parts, int part, int64_t* begin, int64_t* size) {
    if (count < 0 || n_parts <= 0 || part < 0 || part >= n_parts || !begin || !size) return RQ_ERR_INVALID_ARG;
    rq::shard_range(count, n_parts, part, begin, size);
    return RQ_OK;
}

rq_status rq_sharded_create(int n_parts, const int* devices, const rq_scene_t* scenes, int64_t max_rays,
                            rq_sharded_t* out) {
    if (!out || n_parts <= 0 || n_parts > 64 || !devices || !scenes || max_rays < 0) return RQ_ERR_INVALID_ARG;
    int n_dev = 0;
    RQ_CUDA(cudaGetDeviceCount(&n_dev));
    for (int k = 0; k < n_parts; ++k) {
        if (!scenes[k] || devices[k] < 0 || devices[k] >= n_dev) return RQ_ERR_INVALID_ARG;
        if (scenes[k]->device != devices[k]) {
            rq::set_last_error("rq_sharded_create: scene of part " + std::to_string(k) + " lives on device " +
                               std::to_string(scenes[k]->device) + ", not " + std::to_string(devices[k]));
            return RQ_ERR_INVALID_ARG;
        }
        if (scenes[k]->kind != scenes[0]->kind) return RQ_ERR_INVALID_ARG;
    }
    rq_sharded* s = new rq_sharded();
    s->max_rays = max_rays;
    s->capacity = (max_rays + n_parts - 1) / n_parts;
    s->parts.resize(n_parts);
    rq_status st = RQ_OK;
    for (int k = 0; k < n_parts && st == RQ_OK; ++k) {
        auto& p = s->parts[k];
        p.device = devices[k];
        p.scene = scenes[k];
        DeviceGuard g(p.device);
        if (g.err != cudaSuccess) { st = cuda_fail(g.err, "rq_sharded_create: cudaSetDevice"); break; }
        st = rq_ctx_create(&p.ctx);
        if (st != RQ_OK) break;
        cudaError_t e = cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p.ready, cudaEventDisableTiming);
        if (e == cudaSuccess && k > 0 && s->capacity > 0) {
            e = cudaMalloc(&p.rays, (size_t)s->capacity * sizeof(rq_ray));
            if (e == cudaSuccess) e = cudaMalloc(&p.hits, (size_t)s->capacity * sizeof(rq_hit));
        }
        if (e != cudaSuccess) st = cuda_fail(e, "rq_sharded_create");
    }
    if (st != RQ_OK) {
        destroy_parts(s);
        delete s;
        return st;
    }
    *out = s;
    return RQ_OK;
}

rq_status rq_sharded_trace(rq_sharded_t s, const rq_ray* rays, rq_hit* hits, int64_t count, rq_query query,
                           const rq_launch* launch, void* stream) {
    if (!s || count < 0 || (count > 0 && (!rays || !hits))) return RQ_ERR_INVALID_ARG;
    if (query != RQ_CLOSEST && query != RQ_ANY) return RQ_ERR_INVALID_ARG;
    if (count > s->max_rays) {
        rq::set_last_error("rq_sharded_trace: " + std::to_string(count) + " rays exceed the " +
                           std::to_string(s->max_rays) + " the shards were created for");
        return RQ_ERR_INVALID_ARG;
    }
    if (count == 0) return RQ_OK;
    const int n = (int)s->parts.size();
    const int home = s->parts[0].device;
    // The caller's rays are ready on `stream` (home device): every part
    // starts after it.
    {
        DeviceGuard g(home);
        if (g.err != cudaSuccess) return cuda_fail(g.err, "rq_sharded_trace: cudaSetDevice");
        RQ_CUDA(cudaEventRecord(s->parts[0].ready, (cudaStream_t)stream));
    }
    rq_status first_err = RQ_OK;
    for (int k = 0; k < n; ++k) {
        auto& p = s->parts[k];
        int64_t b = 0, m = 0;
        rq::shard_range(count, n, k, &b, &m);
        if (m == 0) continue;
        DeviceGuard g(p.device);
        if (g.err != cudaSuccess) return cuda_fail(g.err, "rq_sharded_trace: cudaSetDevice");
        RQ_CUDA(cudaStreamWaitEvent(p.stream, s->parts[0].ready, 0));
        rq_status st;
        if (k == 0) {
            st = rq_trace(p.ctx, p.scene, rays + b, hits + b, m, query, launch, p.stream);
        } else {
            RQ_CUDA(cudaMemcpyPeerAsync(p.rays, p.device, rays + b, home, (size_t)m * sizeof(rq_ray), p.stream));
            st = rq_trace(p.ctx, p.scene, p.rays, p.hits, m, query, launch, p.stream);
            if (st == RQ_OK)
                RQ_CUDA(cudaMemcpyPeerAsync(hits + b, home, p.hits, p.device, (size_t)m * sizeof(rq_hit), p.stream));
        }
        if (st != RQ_OK && first_err == RQ_OK) first_err = st;
    }
    // Wait for every part and collect the kernels' error words.
    for (int k = 0; k < n; ++k) {
        auto& p = s->parts[k];
        DeviceGuard g(p.device);
        if (g.err != cudaSuccess) return cuda_fail(g.err, "rq_sharded_trace: cudaSetDevice");
        const rq_status st = rq_ctx_check(p.ctx, p.stream);
        if (st != RQ_OK && first_err == RQ_OK) first_err = st;
    }
    return first_err;
}

rq_status rq_sharded_destroy(rq_sharded_t s) {
    if (!s) return RQ_ERR_INVALID_ARG;
    for (auto& p : s->parts) {
        DeviceGuard g(p.device);
        if (p.stream) cudaStreamSynchronize(p.stream);
    }
    destroy_parts(s);
    delete s;
    return RQ_OK;
}

}  // extern "C"
