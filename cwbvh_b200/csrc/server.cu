// Continuous-batching AO bake server.
//
// Requests queue in arrival order.  A ray request is (scene id, host rays,
// host hit buffer); a bake request is (scene id, host surfels, rays per
// surfel, host AO buffer): its rays are generated on the device and its
// occluded rays counted per surfel in the trace epilogue, so only the surfels
// cross PCIe in and one float per surfel comes back.
//
// Memory.  The HBM budget is one device pool, allocated when the server is
// created; every request buffer lives in it.  A request is cut into pieces
// of at most max_batch_rays rays (whole surfels for bake requests) that each
// fit the pool, so no request is refused for its size: pieces of one request
// may run in different launches, and the request completes when its last
// piece has.  Admission is by bytes: a piece is admitted when the pool can
// give it its buffers (first fit, 256-B aligned), and gives them back when
// its launch has finished, so the bytes in use never exceed the budget and
// queued pieces wait while the budget is taken.
//
// Launches.  A dispatcher thread owns `streams` workers.  Whenever a worker
// is free, it admits the oldest queued pieces (arrival order, up to
// max_batch_rays rays in all) whose buffers the pool can give, copies their
// inputs in, traces all of them in one persistent batch launch and copies the
// results back -- all on the worker's stream -- so batches on different
// workers overlap on the device (the next batch's blocks start as the
// previous one drains) and copies overlap traces.  Pieces arriving meanwhile
// are admitted into the next free worker.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
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
    bool deferred_copy = false;  // pageable destination: copied after the stream finishes
    int pieces_left = 0;
    int pieces_started = 0;
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    int32_t batch = -1;          // launch of the request's first piece
    rq_status status = RQ_OK;
    enum State { kQueued, kRunning, kDone } state = kQueued;
};

// A contiguous part of a request: rays [first, first + n) of a ray request,
// or surfels [first, first + n) of a bake request.
struct Piece {
    Req* req = nullptr;
    int64_t first = 0;
    int64_t n = 0;
    int64_t rays = 0;        // rays traced
    int64_t bytes = 0;       // pool bytes while admitted
    int64_t off = -1;        // pool offset while admitted
    void* dev_out = nullptr;
};

int64_t ray_piece_bytes(int64_t n) {
    return align256(n * (int64_t)sizeof(rq::Ray)) + align256(n * (int64_t)sizeof(rq::Hit));
}
int64_t bake_piece_bytes(int64_t n, int spp, bool radius) {
    return 2 * align256(16 * n) + (radius ? align256(4 * n) : 0) + align256(4 * n) +
           align256(n * spp * (int64_t)sizeof(rq::Ray));
}

// First-fit allocator over the server's device pool (offsets, 256-B units).
struct Pool {
    char* base = nullptr;
    int64_t size = 0;
    std::map<int64_t, int64_t> free_;  // offset -> length
    int64_t in_use = 0, peak = 0;

    void reset(char* b, int64_t n) {
        base = b;
        size = n;
        free_.clear();
        if (n > 0) free_[0] = n;
    }
    int64_t alloc(int64_t n) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const int64_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > n) free_[off + n] = len - n;
            in_use += n;
            peak = std::max(peak, in_use);
            return off;
        }
        return -1;
    }
    void release(int64_t off, int64_t n) {
        in_use -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

// Occluded-ray counts of a bake request turned into AO fractions in place.
__global__ void counts_to_ao_kernel(uint32_t* counts, int64_t n, int spp) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) reinterpret_cast<float*>(counts)[i] = (float)counts[i] / (float)spp;
}

struct Worker {
    cudaStream_t stream = nullptr;
    rq_ctx* ctx = nullptr;
    rq::TraceItem* d_items = nullptr;
    rq::TraceItem* h_items = nullptr;  // pinned
    std::vector<Piece*> inflight;
    bool busy = false;
    bool finished = false;  // set by the stream callback
};

constexpr int kMaxItems = 4096;

}  // namespace

struct rq_server {
    rq_server_params params{};
    int64_t cap = 0;          // rays per launch (and per piece)
    char* d_pool = nullptr;
    Pool pool;
    int64_t admission_waits = 0;  // times the oldest queued piece waited for pool bytes
    int64_t pieces_total = 0;
    rq_launch launch{};
    rq_bvh_kind kind = RQ_BVH_CWBVH;
    std::vector<rq_scene*> scenes;
    std::mutex mu;
    std::condition_variable cv;       // dispatcher wake-ups
    std::condition_variable cv_done;  // request completions
    std::deque<Piece*> pending;
    std::unordered_map<uint64_t, Req*> reqs;
    uint64_t next_ticket = 1;
    int32_t next_batch = 0;
    std::vector<Worker> workers;
    std::thread dispatcher;
    bool stop = false;
    rq_status fatal = RQ_OK;

    void run();
    void launch_batch(Worker& w, std::vector<Piece*>& batch, int32_t batch_id);
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

void rq_server::launch_batch(Worker& w, std::vector<Piece*>& batch, int32_t batch_id) {
    rq_status st = RQ_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == RQ_OK) st = rq::cuda_fail(e, "rq_server batch");
    };
    int64_t ray_begin = 0;
    for (size_t k = 0; k < batch.size(); ++k) {
        Piece* pc = batch[k];
        Req* r = pc->req;
        char* base = d_pool + pc->off;
        int64_t off = 0;
        rq::TraceItem it;
        if (!r->bake) {
            rq::Ray* d_rays = reinterpret_cast<rq::Ray*>(base + off);
            off += align256(pc->n * (int64_t)sizeof(rq::Ray));
            rq::Hit* d_hits = reinterpret_cast<rq::Hit*>(base + off);
            ok(cudaMemcpyAsync(d_rays, r->host_rays + pc->first, (size_t)pc->n * sizeof(rq::Ray),
                               cudaMemcpyHostToDevice, w.stream));
            it = rq::scene_item(scenes[r->scene], (const rq_ray*)d_rays, (rq_hit*)d_hits, pc->n);
            pc->dev_out = d_hits;
        } else {
            const int64_t n = pc->n;
            float* d_pos = reinterpret_cast<float*>(base + off);
            off += align256(16 * n);
            float* d_nrm = reinterpret_cast<float*>(base + off);
            off += align256(16 * n);
            float* d_rad = nullptr;
            if (r->host_radius) {
                d_rad = reinterpret_cast<float*>(base + off);
                off += align256(4 * n);
            }
            uint32_t* d_counts = reinterpret_cast<uint32_t*>(base + off);
            off += align256(4 * n);
            rq_ray* d_rays = reinterpret_cast<rq_ray*>(base + off);
            ok(cudaMemcpyAsync(d_pos, r->host_pos + 4 * pc->first, (size_t)(16 * n), cudaMemcpyHostToDevice,
                               w.stream));
            ok(cudaMemcpyAsync(d_nrm, r->host_nrm + 4 * pc->first, (size_t)(16 * n), cudaMemcpyHostToDevice,
                               w.stream));
            if (d_rad)
                ok(cudaMemcpyAsync(d_rad, r->host_radius + pc->first, (size_t)(4 * n), cudaMemcpyHostToDevice,
                                   w.stream));
            ok(cudaMemsetAsync(d_counts, 0, (size_t)(4 * n), w.stream));
            if (st == RQ_OK)
                st = rq::aorays_launch(d_pos, d_nrm, d_rad, n, r->spp, pc->first * r->spp, r->seed, r->tmin, r->tmax,
                                       r->offset_scale, d_rays, w.stream);
            it = rq::scene_item(scenes[r->scene], d_rays, nullptr, pc->rays);
            it.ao_counts = d_counts;
            it.ao_spp = r->spp;
            pc->dev_out = d_counts;
        }
        it.ray_begin = ray_begin;
        ray_begin += pc->rays;
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
    for (Piece* pc : batch) {
        Req* r = pc->req;
        if (r->bake && st == RQ_OK) {
            counts_to_ao_kernel<<<(unsigned)((pc->n + 255) / 256), 256, 0, w.stream>>>((uint32_t*)pc->dev_out, pc->n,
                                                                                       r->spp);
            ok(cudaGetLastError());
        }
        const int64_t out_elem = r->bake ? 4 : (int64_t)sizeof(rq::Hit);
        if (st == RQ_OK && !r->deferred_copy)
            ok(cudaMemcpyAsync(static_cast<char*>(r->host_out) + pc->first * out_elem, pc->dev_out,
                               (size_t)(pc->n * out_elem), cudaMemcpyDeviceToHost, w.stream));
    }
    if (st != RQ_OK) {
        std::lock_guard<std::mutex> lk(mu);
        for (Piece* pc : batch)
            if (pc->req->status == RQ_OK) pc->req->status = st;
    }
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
    const rq_status kst = rq_ctx_check(w.ctx, w.stream);
    std::vector<rq_status> copy_st(w.inflight.size(), RQ_OK);
    for (size_t k = 0; k < w.inflight.size(); ++k) {
        Piece* pc = w.inflight[k];
        Req* r = pc->req;
        const int64_t out_elem = r->bake ? 4 : (int64_t)sizeof(rq::Hit);
        if (r->deferred_copy &&
            cudaMemcpy(static_cast<char*>(r->host_out) + pc->first * out_elem, pc->dev_out,
                       (size_t)(pc->n * out_elem), cudaMemcpyDeviceToHost) != cudaSuccess)
            copy_st[k] = rq::cuda_fail(cudaGetLastError(), "rq_server: result copy");
    }
    const double t = now_ms();
    {
        std::lock_guard<std::mutex> lk(mu);
        for (size_t k = 0; k < w.inflight.size(); ++k) {
            Piece* pc = w.inflight[k];
            Req* r = pc->req;
            pool.release(pc->off, pc->bytes);
            if (r->status == RQ_OK) r->status = copy_st[k] != RQ_OK ? copy_st[k] : kst;
            if (--r->pieces_left == 0) {
                r->done_ms = t;
                r->state = Req::kDone;
            }
            delete pc;
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
    bool blocked = false;  // the oldest queued piece waits for pool bytes
    for (;;) {
        cv.wait(lk, [&] {
            bool any_busy = false;
            for (auto& w : workers) {
                if (w.busy && w.finished) return true;
                if (!stop && !w.busy && !pending.empty() && !blocked) return true;
                any_busy |= w.busy;
            }
            return stop && !any_busy;
        });
        // Completed batches first: they give their bytes back to the pool.
        for (auto& w : workers)
            if (w.busy && w.finished) {
                lk.unlock();
                finalize(w);
                lk.lock();
                blocked = false;
            }
        if (stop) {
            bool any_busy = false;
            for (auto& w : workers) any_busy |= w.busy;
            if (!any_busy) break;
            continue;  // wait for the in-flight batches to complete
        }
        for (auto& w : workers) {
            if (w.busy || pending.empty() || blocked) continue;
            std::vector<Piece*> batch;
            int64_t rays = 0;
            while (!pending.empty() && (int)batch.size() < kMaxItems) {
                Piece* pc = pending.front();
                if (!batch.empty() && rays + pc->rays > cap) break;
                const int64_t off = pool.alloc(pc->bytes);
                if (off < 0) {
                    // Arrival order is kept: later pieces wait behind this one.
                    blocked = true;
                    ++admission_waits;
                    break;
                }
                pc->off = off;
                pending.pop_front();
                rays += pc->rays;
                batch.push_back(pc);
            }
            if (batch.empty()) continue;
            const double t = now_ms();
            const int32_t id = next_batch++;
            for (Piece* pc : batch) {
                Req* r = pc->req;
                if (r->pieces_started++ == 0) {
                    r->state = Req::kRunning;
                    r->start_ms = t;
                    r->batch = id;
                }
            }
            w.busy = true;
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
    const int streams = params->streams > 0 ? params->streams : 3;
    const int64_t budget = params->hbm_budget_bytes / 256 * 256;
    // Rays per launch: by default every worker can hold a full launch at
    // once; never more than one piece of that size fits the pool.
    int64_t cap = budget / (48 * (int64_t)streams);
    if (params->max_batch_rays > 0) cap = params->max_batch_rays;
    cap = std::min(cap, (budget - 512) / 48);
    if (cap <= 0) return RQ_ERR_INVALID_ARG;
    rq_server* s = new rq_server();
    s->params = *params;
    s->params.streams = streams;
    s->params.hbm_budget_bytes = budget;
    s->cap = cap;
    cudaError_t e = cudaMalloc(&s->d_pool, (size_t)budget);
    if (e != cudaSuccess) {
        delete s;
        return rq::cuda_fail(e, "rq_server_create: the HBM budget's pool");
    }
    s->pool.reset(s->d_pool, budget);
    s->workers.resize(streams);
    rq_status st = RQ_OK;
    for (auto& w : s->workers) {
        if (st != RQ_OK) break;
        e = cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) st = rq_ctx_create(&w.ctx);
        else st = rq::cuda_fail(e, "rq_server_create");
        if (st != RQ_OK) break;
        e = cudaMalloc(&w.d_items, kMaxItems * sizeof(rq::TraceItem));
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

// Cuts a request into pieces (each fits the pool and one launch) and queues
// them in order.  `unit` is rays (ray request) or surfels (bake request).
static rq_status enqueue(rq_server_t s, Req* r, int64_t units, int64_t units_per_piece) {
    if (units_per_piece <= 0) {
        delete r;
        return RQ_ERR_BUDGET;
    }
    std::vector<Piece*> pieces;
    for (int64_t first = 0; first < units; first += units_per_piece) {
        Piece* pc = new Piece();
        pc->req = r;
        pc->first = first;
        pc->n = std::min(units_per_piece, units - first);
        pc->rays = r->bake ? pc->n * r->spp : pc->n;
        pc->bytes = r->bake ? bake_piece_bytes(pc->n, r->spp, r->host_radius != nullptr) : ray_piece_bytes(pc->n);
        pieces.push_back(pc);
    }
    r->pieces_left = (int)pieces.size();
    r->deferred_copy = !is_pinned(r->host_out);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        rq_status st = RQ_OK;
        if (s->stop) st = RQ_ERR_CANCELLED;
        else if (r->scene < 0 || r->scene >= (int32_t)s->scenes.size()) st = RQ_ERR_NOT_FOUND;
        if (st != RQ_OK) {
            for (Piece* pc : pieces) delete pc;
            delete r;
            return st;
        }
        r->ticket = s->next_ticket++;
        r->submit_ms = now_ms();
        s->reqs[r->ticket] = r;
        for (Piece* pc : pieces) s->pending.push_back(pc);
        s->pieces_total += (int64_t)pieces.size();
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
    const rq_status st = enqueue(s, r, count, s->cap);
    if (st == RQ_OK) *ticket = r->ticket;
    return st;
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
    // Whole surfels per piece: at most one launch of rays, and buffers that
    // fit the pool.
    int64_t per = std::min<int64_t>(n_surfels, s->cap / spp);
    const int64_t per_surfel = 40 + (host_radius ? 4 : 0) + 32 * (int64_t)spp;
    per = std::min<int64_t>(per, (s->params.hbm_budget_bytes - 5 * 256) / per_surfel);
    while (per > 0 && bake_piece_bytes(per, spp, host_radius != nullptr) > s->params.hbm_budget_bytes) --per;
    const rq_status st = enqueue(s, r, n_surfels, per);
    if (st == RQ_OK) *ticket = r->ticket;
    return st;
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
        // Not started: all of its pieces are still queued.
        for (auto p = s->pending.begin(); p != s->pending.end();) {
            if ((*p)->req == r) {
                delete *p;
                p = s->pending.erase(p);
            } else {
                ++p;
            }
        }
        r->pieces_left = 0;
        r->status = RQ_ERR_CANCELLED;
        r->state = Req::kDone;
        r->done_ms = now_ms();
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    return RQ_OK;
}

rq_status rq_server_memory(rq_server_t s, rq_server_memory_stats* out) {
    if (!s || !out) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    out->pool_bytes = s->pool.size;
    out->in_use_bytes = s->pool.in_use;
    out->peak_in_use_bytes = s->pool.peak;
    out->admission_waits = s->admission_waits;
    out->pieces = s->pieces_total;
    out->max_batch_rays = s->cap;
    return RQ_OK;
}

rq_status rq_server_destroy(rq_server_t s) {
    if (!s) return RQ_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        const double t = now_ms();
        for (Piece* pc : s->pending) {
            Req* r = pc->req;
            r->status = RQ_ERR_CANCELLED;
            if (--r->pieces_left == 0) {  // pieces still running finish it otherwise
                r->state = Req::kDone;
                r->done_ms = t;
            }
            delete pc;
        }
        s->pending.clear();
    }
    s->cv.notify_all();
    s->cv_done.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    for (auto& w : s->workers) {
        if (w.stream) cudaStreamSynchronize(w.stream);
        if (w.ctx) rq_ctx_destroy(w.ctx);
        cudaFree(w.d_items);
        if (w.h_items) cudaFreeHost(w.h_items);
        if (w.stream) cudaStreamDestroy(w.stream);
    }
    cudaFree(s->d_pool);
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return RQ_OK;
}

}  // extern "C"
