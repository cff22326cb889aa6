// Continuous-batching AO bake server.
//
// Requests (scene id, host rays, host hit buffer) queue in arrival order.  A
// dispatcher thread owns `streams` workers; each worker has device ray/hit
// arenas of max_batch_rays rays (48 B per ray), so the HBM taken by ray/hit
// buffers never exceeds streams x max_batch_rays x 48 <= hbm_budget_bytes.
// Whenever a worker is free, the dispatcher admits the oldest queued requests
// that fit its arena, copies their rays in, traces all of them in one
// persistent batch launch and copies the hits back -- all on the worker's
// stream -- so batches on different workers overlap on the device (the next
// batch's blocks start as the previous one drains) and copies overlap traces.
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

struct Req {
    uint64_t ticket = 0;
    int32_t scene = 0;
    const rq_ray* host_rays = nullptr;
    rq_hit* host_hits = nullptr;
    int64_t count = 0;
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    int32_t batch = -1;
    rq_status status = RQ_OK;
    enum State { kQueued, kRunning, kDone } state = kQueued;
    int64_t offset = 0;         // in the worker arena
    bool deferred_copy = false;  // pageable destination: copied after the stream finishes
};

struct Worker {
    cudaStream_t stream = nullptr;
    rq_ctx* ctx = nullptr;
    rq::Ray* d_rays = nullptr;
    rq::Hit* d_hits = nullptr;
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
    int64_t cap = 0;
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
    int64_t off = 0;
    for (size_t k = 0; k < batch.size(); ++k) {
        Req* r = batch[k];
        r->offset = off;
        r->batch = batch_id;
        if (cudaMemcpyAsync(w.d_rays + off, r->host_rays, (size_t)r->count * sizeof(rq::Ray), cudaMemcpyHostToDevice,
                            w.stream) != cudaSuccess)
            st = RQ_ERR_CUDA;
        rq::TraceItem it = rq::scene_item(scenes[r->scene], (const rq_ray*)(w.d_rays + off), (rq_hit*)(w.d_hits + off),
                                          r->count);
        it.ray_begin = off;
        w.h_items[k] = it;
        off += r->count;
    }
    if (st == RQ_OK && cudaMemcpyAsync(w.d_items, w.h_items, batch.size() * sizeof(rq::TraceItem),
                                       cudaMemcpyHostToDevice, w.stream) != cudaSuccess)
        st = RQ_ERR_CUDA;
    if (st == RQ_OK) st = rq::reset_counter(w.ctx, w.stream);
    if (st == RQ_OK) {
        rq::TraceParams p = rq::base_params(w.ctx, launch);
        p.single = w.h_items[0];
        p.items = w.d_items;
        p.n_items = (int)batch.size();
        p.total_rays = off;
        st = rq::launch_trace(kind, params.query, launch, true, false, p, w.stream);
    }
    for (Req* r : batch) {
        r->deferred_copy = !is_pinned(r->host_hits);
        if (st == RQ_OK && !r->deferred_copy &&
            cudaMemcpyAsync(r->host_hits, w.d_hits + r->offset, (size_t)r->count * sizeof(rq::Hit),
                            cudaMemcpyDeviceToHost, w.stream) != cudaSuccess)
            st = RQ_ERR_CUDA;
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
            cudaMemcpy(r->host_hits, w.d_hits + r->offset, (size_t)r->count * sizeof(rq::Hit),
                       cudaMemcpyDeviceToHost) != cudaSuccess)
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
            int64_t rays = 0;
            while (!pending.empty() && (int)batch.size() < kMaxItems && rays + pending.front()->count <= cap) {
                Req* r = pending.front();
                pending.pop_front();
                rays += r->count;
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
        e = cudaMalloc(&w.d_rays, (size_t)cap * sizeof(rq::Ray));
        if (e == cudaSuccess) e = cudaMalloc(&w.d_hits, (size_t)cap * sizeof(rq::Hit));
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

rq_status rq_server_submit(rq_server_t s, int32_t scene_id, const rq_ray* host_rays, rq_hit* host_hits, int64_t count,
                           uint64_t* ticket) {
    if (!s || !host_rays || !host_hits || count <= 0 || !ticket) return RQ_ERR_INVALID_ARG;
    Req* r = new Req();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return RQ_ERR_CANCELLED;
        }
        if (scene_id < 0 || scene_id >= (int32_t)s->scenes.size()) {
            delete r;
            return RQ_ERR_NOT_FOUND;
        }
        if (count > s->cap) {
            delete r;
            return RQ_ERR_BUDGET;
        }
        r->ticket = s->next_ticket++;
        r->scene = scene_id;
        r->host_rays = host_rays;
        r->host_hits = host_hits;
        r->count = count;
        r->submit_ms = now_ms();
        s->reqs[r->ticket] = r;
        s->pending.push_back(r);
        *ticket = r->ticket;
    }
    s->cv.notify_all();
    return RQ_OK;
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
        cudaFree(w.d_rays);
        cudaFree(w.d_hits);
        cudaFree(w.d_items);
        if (w.h_items) cudaFreeHost(w.h_items);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return RQ_OK;
}

}  // extern "C"
