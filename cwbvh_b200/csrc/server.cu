// Continuous-batching AO bake server.
//
// Requests queue in arrival order.  A ray request is (scene id, host rays,
// host hit buffer); a bake request is (scene id, host surfels, rays per
// surfel, host AO buffer): its rays are generated on the device and its
// occluded rays counted per surfel in the trace epilogue, so only the surfels
// cross PCIe in and one float per surfel comes back.  A dispatcher thread
// owns `streams` workers; each worker has one device arena of max_batch_rays
// x 48 B, so the HBM taken by request buffers never exceeds
// streams x max_batch_rays x 48 <= hbm_budget_bytes.  Whenever a worker is
// free, the dispatcher admits the oldest queued requests whose buffers fit
// its arena, copies their inputs in, traces all of them in one persistent
// batch launch and copies the results back -- all on the worker's stream --
// so batches on different workers overlap on the device (the next batch's
// blocks start as the previous one drains) and copies overlap traces.
// Requests arriving meanwhile are admitted into the next free worker.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "runtime.h"

namespace {

double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

bool is_pinned(const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

int64_t align256(int64_t b) { return (b + 255) & ~(int64_t)255; }

struct Req {
    uint64_t ticket = 0;
    int32_t scene = 0;
    const rq_ray* host_rays = nullptr;
    int64_t count = 0;           // rays
    // bake requests: surfels in, AO out
    bool bake = false;
    const float* host_pos = nullptr;
    const float* host_nrm = nullptr;
    const float* host_radius = nullptr;
    int64_t n_surfels = 0;
    int spp = 0;
    uint64_t seed = 0;
    float tmin = 0.f, tmax = 0.f, offset_scale = 0.f;
    // result: hits (ray request) or AO per surfel (bake request)
    void* host_out = nullptr;
    void* dev_out = nullptr;
    int64_t out_bytes = 0;
    int64_t arena_bytes = 0;     // device bytes the request occupies while running
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    int32_t batch = -1;
    rq_status status = RQ_OK;
    enum State { kQueued, kRunning, kDone } state = kQueued;
    bool deferred_copy = false;  // pageable destination: copied after the stream finishes
};

// Occluded-ray counts of a bake request turned into AO fractions in place.
__global__ void counts_to_ao_kernel(uint32_t* counts, int64_t n, int spp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) reinterpret_cast<float*>(counts)[i] = (float)counts[i] / (float)spp;
}

struct Worker {
    cudaStream_t stream = nullptr;
    rq_ctx* ctx = nullptr;
    char* d_arena = nullptr;
    rq::TraceItem* d_items = nullptr;
    rq::TraceItem* h_items = nullptr;  // pinned
    std::vector<Req*> inflight;
    bool busy = false;
    bool finished = false;  // set by the stream callback
};

constexpr int kMaxItems = 4096;

}  // namespace

struct rq_server {
    rq_server_params params{};
    int64_t cap = 0;          // rays of a ray request that fill an arena
    int64_t arena_bytes = 0;  // per worker
    rq_launch launch{};
    rq_bvh_kind kind = RQ_BVH_CWBVH;
    std::vector<rq_scene*> scenes;
    std::mutex mu;
    std::condition_variable cv;       // dispatcher wake-ups
    std::condition_variable cv_done;  // request completions
    std::deque<Req*> pending;
    std::unordered_map<uint64_t, Req*> reqs;
    uint64_t next_ticket = 1;
    int32_t next_batch = 0;
    std::vector<Worker> workers;
    std::thread dispatcher;
    bool stop = false;
    rq_status fatal = RQ_OK;

    void run();
    void launch_batch(Worker& w, std::vector<Req*>& batch, int32_t batch_id);
    void finalize(Worker& w);
};

static void CUDART_CB worker_done(void* user) {
    auto* pair = static_cast<std::pair<rq_server*, Worker*>*>(user);
    {
        std::lock_guard<std::mutex> lk(pair->first->mu);
        pair->second->finished = true;
    }
    pair->first->cv.notify_all();
    delete pair;
}

void rq_server::launch_batch(Worker& w, std::vector<Req*>& batch, int32_t batch_id) {
    rq_status st = RQ_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == RQ_OK) st = rq::cuda_fail(e, "rq_server batch");
    };
    int64_t off = 0, ray_begin = 0;
    for (size_t k = 0; k < batch.size(); ++k) {
        Req* r = batch[k];
        r->batch = batch_id;
        rq::TraceItem it;
        if (!r->bake) {
            rq::Ray* d_rays = reinterpret_cast<rq::Ray*>(w.d_arena + off);
            off += align256(r->count * (int64_t)sizeof(rq::Ray));
            rq::Hit* d_hits = reinterpret_cast<rq::Hit*>(w.d_arena + off);
            off += align256(r->count * (int64_t)sizeof(rq::Hit));
            ok(cudaMemcpyAsync(d_rays, r->host_rays, (size_t)r->count * sizeof(rq::Ray), cudaMemcpyHostToDevice,
                               w.stream));
            it = rq::scene_item(scenes[r->scene], (const rq_ray*)d_rays, (rq_hit*)d_hits, r->count);
            r->dev_out = d_hits;
        } else {
            const int64_t n = r->n_surfels;
            float* d_pos = reinterpret_cast<float*>(w.d_arena + off);
            off += align256(16 * n);
            float* d_nrm = reinterpret_cast<float*>(w.d_arena + off);
            off += align256(16 * n);
            float* d_rad = nullptr;
            if (r->host_radius) {
                d_rad = reinterpret_cast<float*>(w.d_arena + off);
                off += align256(4 * n);
            }
            uint32_t* d_counts = reinterpret_cast<uint32_t*>(w.d_arena + off);
            off += align256(4 * n);
            rq_ray* d_rays = reinterpret_cast<rq_ray*>(w.d_arena + off);
            off += align256(r->count * (int64_t)sizeof(rq::Ray));
            ok(cudaMemcpyAsync(d_pos, r->host_pos, (size_t)(16 * n), cudaMemcpyHostToDevice, w.stream));
            ok(cudaMemcpyAsync(d_nrm, r->host_nrm, (size_t)(16 * n), cudaMemcpyHostToDevice, w.stream));
            if (d_rad) ok(cudaMemcpyAsync(d_rad, r->host_radius, (size_t)(4 * n), cudaMemcpyHostToDevice, w.stream));
            ok(cudaMemsetAsync(d_counts, 0, (size_t)(4 * n), w.stream));
            if (st == RQ_OK)
                st = rq_aorays(d_pos, d_nrm, d_rad, n, r->spp, r->seed, r->tmin, r->tmax, r->offset_scale, d_rays,
                               w.stream);
            it = rq::scene_item(scenes[r->scene], d_rays, nullptr, r->count);
            it.ao_counts = d_counts;
            it.ao_spp = r->spp;
            r->dev_out = d_counts;
        }
        it.ray_begin = ray_begin;
        ray_begin += r->count;
        w.h_items[k] = it;
    }
    if (st == RQ_OK)
        ok(cudaMemcpyAsync(w.d_items, w.h_items, batch.size() * sizeof(rq::TraceItem), cudaMemcpyHostToDevice,
                           w.stream));
    if (st == RQ_OK) st = rq::reset_counter(w.ctx, w.stream);
    if (st == RQ_OK) {
        rq::TraceParams p = rq::base_params(w.ctx, launch);
        p.single = w.h_items[0];
        p.items = w.d_items;
        p.n_items = (int)batch.size();
        p.total_rays = ray_begin;
        st = rq::launch_trace(kind, params.query, launch, true, false, p, w.stream);
    }
    for (Req* r : batch) {
        if (r->bake && st == RQ_OK) {
            counts_to_ao_kernel<<<(unsigned)((r->n_surfels + 255) / 256), 256, 0, w.stream>>>(
                (uint32_t*)r->dev_out, r->n_surfels, r->spp);
            ok(cudaGetLastError());
        }
        r->deferred_copy = !is_pinned(r->host_out);
        if (st == RQ_OK && !r->deferred_copy)
            ok(cudaMemcpyAsync(r->host_out, r->dev_out, (size_t)r->out_bytes, cudaMemcpyDeviceToHost, w.stream));
    }
    for (Req* r : batch) r->status = st;
    w.inflight = batch;
    w.finished = false;
    auto* pair = new std::pair<rq_server*, Worker*>(this, &w);
    if (cudaLaunchHostFunc(w.stream, worker_done, pair) != cudaSuccess) {
        delete pair;
        cudaStreamSynchronize(w.stream);
        std::lock_guard<std::mutex> lk(mu);
        w.finished = true;
    }
}

void rq_server::finalize(Worker& w) {
    // Called without the lock; the stream has completed.
    rq_status kst = rq_ctx_check(w.ctx, w.stream);
    for (Req* r : w.inflight) {
        if (r->status == RQ_OK && r->deferred_copy &&
            cudaMemcpy(r->host_out, r->dev_out, (size_t)r->out_bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
            r->status = RQ_ERR_CUDA;
        if (r->status == RQ_OK) r->status = kst;
    }
    const double t = now_ms();
    {
        std::lock_guard<std::mutex> lk(mu);
        for (Req* r : w.inflight) {
            r->done_ms = t;
            r->state = Req::kDone;
        }
        w.inflight.clear();
        w.busy = false;
        w.finished = false;
    }
    cv_done.notify_all();
    cv.notify_all();
}

void rq_server::run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        cv.wait(lk, [&] {
            bool any_busy = false;
            for (auto& w : workers) {
                if (w.busy && w.finished) return true;
                if (!stop && !w.busy && !pending.empty()) return true;
                any_busy |= w.busy;
            }
            return stop && !any_busy;
        });
        // Completed batches first: they free arenas for the queue.
        for (auto& w : workers)
            if (w.busy && w.finished) {
                lk.unlock();
                finalize(w);
                lk.lock();
            }
        if (stop) {
            bool any_busy = false;
            for (auto& w : workers) any_busy |= w.busy;
            if (!any_busy) break;
            continue;  // wait for the in-flight batches to complete
        }
        for (auto& w : workers) {
            if (w.busy || pending.empty()) continue;
            std::vector<Req*> batch;
            int64_t bytes = 0;
            while (!pending.empty() && (int)batch.size() < kMaxItems &&
                   bytes + pending.front()->arena_bytes <= arena_bytes) {
                Req* r = pending.front();
                pending.pop_front();
                bytes += r->arena_bytes;
                batch.push_back(r);
            }
            if (batch.empty()) continue;
            const double t = now_ms();
            for (Req* r : batch) {
                r->state = Req::kRunning;
                r->start_ms = t;
            }
            w.busy = true;
            const int32_t id = next_batch++;
            lk.unlock();
            launch_batch(w, batch, id);
            lk.lock();
        }
    }
}

extern "C" {

rq_status rq_server_create(const rq_server_params* params, rq_server_t* out) {
    if (!params || !out || params->hbm_budget_bytes <= 0) return RQ_ERR_INVALID_ARG;
    if (params->query != RQ_CLOSEST && params->query != RQ_ANY) return RQ_ERR_INVALID_ARG;
    rq_server* s = new rq_server();
    s->params = *params;
    const int streams = params->streams > 0 ? params->streams : 3;
    s->params.streams = streams;
    int64_t cap = params->hbm_budget_bytes / (48 * (int64_t)streams);
    if (params->max_batch_rays > 0) cap = std::min(cap, params->max_batch_rays);
    s->cap = cap;
    s->arena_bytes = 48 * cap + 512;  // + two 256-B alignment pads: a ray request of `cap` rays fits
    if (cap <= 0) {
        delete s;
        return RQ_ERR_INVALID_ARG;
    }
    s->workers.resize(streams);
    rq_status st = RQ_OK;
    for (auto& w : s->workers) {
        if (st != RQ_OK) break;
        cudaError_t e = cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) st = rq_ctx_create(&w.ctx);
        else st = rq::cuda_fail(e, "rq_server_create");
        if (st != RQ_OK) break;
        e = cudaMalloc(&w.d_arena, (size_t)s->arena_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&w.d_items, kMaxItems * sizeof(rq::TraceItem));
        if (e == cudaSuccess) e = cudaMallocHost(&w.h_items, kMaxItems * sizeof(rq::TraceItem));
        if (e != cudaSuccess) st = rq::cuda_fail(e, "rq_server_create");
    }
    if (st != RQ_OK) {
        rq_server_destroy(s);
        return st;
    }
    s->dispatcher = std::thread([s] { s->run(); });
    *out = s;
    return RQ_OK;
}

rq_status rq_server_add_scene(rq_server_t s, rq_scene_t scene, int32_t* scene_id) {
    if (!s || !scene || !scene_id) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->scenes.empty()) {
        s->kind = scene->kind;
        s->launch = rq::resolve_launch(scene->kind, s->params.query, &s->params.launch);
    } else if (scene->kind != s->kind) {
        return RQ_ERR_INVALID_ARG;  // one kernel family per server
    }
    *scene_id = (int32_t)s->scenes.size();
    s->scenes.push_back(scene);
    return RQ_OK;
}

static rq_status enqueue(rq_server_t s, Req* r, uint64_t* ticket) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        rq_status st = RQ_OK;
        if (s->stop) st = RQ_ERR_CANCELLED;
        else if (r->scene < 0 || r->scene >= (int32_t)s->scenes.size()) st = RQ_ERR_NOT_FOUND;
        else if (r->arena_bytes > s->arena_bytes) st = RQ_ERR_BUDGET;
        if (st != RQ_OK) {
            delete r;
            return st;
        }
        r->ticket = s->next_ticket++;
        r->submit_ms = now_ms();
        s->reqs[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv.notify_all();
    return RQ_OK;
}

rq_status rq_server_submit(rq_server_t s, int32_t scene_id, const rq_ray* host_rays, rq_hit* host_hits, int64_t count,
                           uint64_t* ticket) {
    if (!s || !host_rays || !host_hits || count <= 0 || !ticket) return RQ_ERR_INVALID_ARG;
    Req* r = new Req();
    r->scene = scene_id;
    r->host_rays = host_rays;
    r->count = count;
    r->host_out = host_hits;
    r->out_bytes = count * (int64_t)sizeof(rq::Hit);
    r->arena_bytes = align256(count * (int64_t)sizeof(rq::Ray)) + align256(count * (int64_t)sizeof(rq::Hit));
    return enqueue(s, r, ticket);
}

rq_status rq_server_submit_bake(rq_server_t s, int32_t scene_id, const float* host_pos, const float* host_nrm,
                                const float* host_radius, int64_t n_surfels, int spp, uint64_t seed, float tmin,
                                float tmax, float offset_scale, float* host_ao, uint64_t* ticket) {
    if (!s || !host_pos || !host_nrm || !host_ao || n_surfels <= 0 || spp <= 0 || !ticket ||
        n_surfels > INT64_MAX / 64 / spp)
        return RQ_ERR_INVALID_ARG;
    if (s->params.query != RQ_ANY) return RQ_ERR_INVALID_ARG;  // AO counts need the any-hit kernels
    Req* r = new Req();
    r->scene = scene_id;
    r->bake = true;
    r->host_pos = host_pos;
    r->host_nrm = host_nrm;
    r->host_radius = host_radius;
    r->n_surfels = n_surfels;
    r->spp = spp;
    r->seed = seed;
    r->tmin = tmin;
    r->tmax = tmax;
    r->offset_scale = offset_scale;
    r->count = n_surfels * spp;
    r->host_out = host_ao;
    r->out_bytes = 4 * n_surfels;
    r->arena_bytes = 2 * align256(16 * n_surfels) + (host_radius ? align256(4 * n_surfels) : 0) +
                     align256(4 * n_surfels) + align256(r->count * (int64_t)sizeof(rq::Ray));
    return enqueue(s, r, ticket);
}

rq_status rq_server_wait(rq_server_t s, uint64_t ticket, int64_t timeout_ms, rq_request_stats* stats) {
    if (!s) return RQ_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return RQ_ERR_NOT_FOUND;
    Req* r = it->second;
    auto done = [&] { return r->state == Req::kDone; };
    if (timeout_ms < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return RQ_ERR_TIMEOUT;
    if (stats) {
        stats->submit_ms = r->submit_ms;
        stats->start_ms = r->start_ms;
        stats->done_ms = r->done_ms;
        stats->rays = r->count;
        stats->batch_id = r->batch;
        stats->status = r->status;
    }
    const rq_status st = r->status;
    s->reqs.erase(it);
    delete r;
    return st;
}

rq_status rq_server_cancel(rq_server_t s, uint64_t ticket) {
    if (!s) return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end() || it->second->state != Req::kQueued) return RQ_ERR_NOT_FOUND;
        Req* r = it->second;
        s->pending.erase(std::find(s->pending.begin(), s->pending.end(), r));
        r->status = RQ_ERR_CANCELLED;
        r->state = Req::kDone;
        r->done_ms = now_ms();
    }
    s->cv_done.notify_all();
    return RQ_OK;
}

rq_status rq_server_destroy(rq_server_t s) {
    if (!s) return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        for (Req* r : s->pending) {
            r->status = RQ_ERR_CANCELLED;
            r->state = Req::kDone;
        }
        s->pending.clear();
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    for (auto& w : s->workers) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        if (w.ctx) rq_ctx_destroy(w.ctx);
        cudaFree(w.d_arena);
        cudaFree(w.d_items);
        if (w.h_items) cudaFreeHost(w.h_items);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return RQ_OK;
}

}  // extern "C"
