// Batched tracing: many (scene, rays, hits) items in one persistent launch,
// with optional Morton sorting of each item's rays and CUDA-graph replay; and
// the launch-shape autotuner with its on-disk cache.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "runtime.h"

struct rq_batch {
    rq_ctx* ctx = nullptr;
    rq_query query = RQ_ANY;
    rq_bvh_kind kind = RQ_BVH_CWBVH;
    rq_launch launch{};
    rq_batch_params params{};
    std::vector<rq::TraceItem> items;  // host copy (ray_begin = global prefix)
    rq::TraceItem* d_items = nullptr;
    int64_t total = 0;
    bool sorted_any = false;
    rq::SortPlan plan;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace rq {

static rq_status batch_enqueue(rq_batch* b, cudaStream_t s) {
    if (b->sorted_any) {
        rq_status st = sort_plan_run(b->plan, s);
        if (st != RQ_OK) return st;
    }
    rq_status st = reset_counter(b->ctx, s);
    if (st != RQ_OK) return st;
    TraceParams p = base_params(b->ctx, b->launch);
    p.single = b->items.empty() ? TraceItem{} : b->items[0];
    p.items = b->d_items;
    p.n_items = (int)b->items.size();
    p.total_rays = b->total;
    return launch_trace(b->kind, b->query, b->launch, true, false, p, s);
}

}  // namespace rq

using namespace rq;

extern "C" {

rq_status rq_batch_create(rq_ctx_t ctx, const rq_batch_item* items, int n_items, rq_query query,
                          const rq_batch_params* params, rq_batch_t* out) {
    if (!ctx || !out || n_items <= 0 || !items) return RQ_ERR_INVALID_ARG;
    if (query != RQ_CLOSEST && query != RQ_ANY) return RQ_ERR_INVALID_ARG;
    const rq_bvh_kind kind = items[0].scene ? items[0].scene->kind : RQ_BVH_CWBVH;
    for (int i = 0; i < n_items; ++i) {
        const rq_batch_item& it = items[i];
        if (!it.scene || it.count < 0 || (it.count > 0 && (!it.rays || !it.hits))) return RQ_ERR_INVALID_ARG;
        if (((uintptr_t)it.rays | (uintptr_t)it.hits) & 15u) return RQ_ERR_INVALID_ARG;  // float4 records
        if (it.scene->kind != kind) return RQ_ERR_INVALID_ARG;  // one kernel family per batch
    }
    rq_batch* b = new rq_batch();
    b->ctx = ctx;
    b->query = query;
    b->kind = kind;
    if (params) b->params = *params;
    else b->params.sort_threshold = -1;
    b->launch = resolve_launch(kind, query, params ? &params->launch : nullptr);

    std::vector<TraceItem> to_sort;
    std::vector<float> bounds;
    std::vector<int> sorted_idx;
    int64_t off = 0;
    for (int i = 0; i < n_items; ++i) {
        TraceItem t = scene_item(items[i].scene, items[i].rays, items[i].hits, items[i].count);
        t.ray_begin = off;
        off += t.count;
        b->items.push_back(t);
        if (b->params.sort_threshold >= 0 && t.count > 0 && t.count >= b->params.sort_threshold) {
            to_sort.push_back(t);
            sorted_idx.push_back(i);
            for (int a = 0; a < 3; ++a) bounds.push_back(items[i].scene->lo[a]);
            for (int a = 0; a < 3; ++a) bounds.push_back(items[i].scene->hi[a]);
        }
    }
    b->total = off;
    rq_status st = RQ_OK;
    if (!to_sort.empty()) {
        st = sort_plan_create(to_sort, bounds, b->plan);
        if (st == RQ_OK) {
            b->sorted_any = true;
            int64_t soff = 0;
            for (size_t k = 0; k < sorted_idx.size(); ++k) {
                TraceItem& t = b->items[sorted_idx[k]];
                t.rays = b->plan.sorted + soff;
                t.perm = b->plan.vals_out + soff;
                soff += t.count;
            }
        }
    }
    if (st == RQ_OK) {
        cudaError_t e = cudaMalloc(&b->d_items, b->items.size() * sizeof(TraceItem));
        if (e == cudaSuccess)
            e = cudaMemcpy(b->d_items, b->items.data(), b->items.size() * sizeof(TraceItem), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) st = cuda_fail(e, "rq_batch_create");
    }
    if (st != RQ_OK) {
        rq_batch_destroy(b);
        return st;
    }
    *out = b;
    return RQ_OK;
}

rq_status rq_batch_run(rq_batch_t b, void* stream) {
    if (!b) return RQ_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->params.use_graph || s == nullptr) return batch_enqueue(b, s);
    if (!b->exec) {
        warm_launch_cache(b->kind, b->query, b->launch, true, false);
        RQ_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        rq_status st = batch_enqueue(b, s);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (st != RQ_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        b->graph = g;
        RQ_CUDA(cudaGraphInstantiate(&b->exec, g, 0));
    }
    RQ_CUDA(cudaGraphLaunch(b->exec, s));
    return RQ_OK;
}

rq_status rq_batch_run_stage(rq_batch_t b, int stage, void* stream) {
    if (!b || stage < 1 || stage > 2) return RQ_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (stage == 1) return b->sorted_any ? sort_plan_run(b->plan, s) : RQ_OK;
    rq_status st = reset_counter(b->ctx, s);
    if (st != RQ_OK) return st;
    TraceParams p = base_params(b->ctx, b->launch);
    p.single = b->items.empty() ? TraceItem{} : b->items[0];
    p.items = b->d_items;
    p.n_items = (int)b->items.size();
    p.total_rays = b->total;
    return launch_trace(b->kind, b->query, b->launch, true, false, p, s);
}

int rq_batch_kernel_count(rq_batch_t b) {
    if (!b) return 0;
    if (b->graph) {
        size_t n = 0;
        if (cudaGraphGetNodes(b->graph, nullptr, &n) != cudaSuccess) return 0;
        std::vector<cudaGraphNode_t> nodes(n);
        if (cudaGraphGetNodes(b->graph, nodes.data(), &n) != cudaSuccess) return 0;
        int k = 0;
        for (auto nd : nodes) {
            cudaGraphNodeType t;
            if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
        }
        return k;
    }
    // Eager: trace kernel, plus Morton keys, the radix sort passes and the gather.
    int k = b->total > 0 ? 1 : 0;
    if (b->sorted_any) k += sort_plan_kernel_count(b->plan);
    return k;
}

int64_t rq_batch_total_rays(rq_batch_t b) { return b ? b->total : 0; }

rq_status rq_batch_destroy(rq_batch_t b) {
    if (!b) return RQ_ERR_INVALID_ARG;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->d_items) cudaFree(b->d_items);
    if (b->sorted_any) sort_plan_destroy(b->plan);
    delete b;
    return RQ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- autotune

namespace rq {

static std::mutex g_tune_mu;

static std::string tune_key(rq_bvh_kind kind, rq_query q, int64_t count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, dev);
    int cls = 0;
    while ((int64_t(1) << (cls + 1)) <= std::max<int64_t>(1, count)) ++cls;
    std::string name(prop.name);
    for (auto& c : name)
        if (c == ' ') c = '_';
    std::ostringstream os;
    os << name << "|" << (kind == RQ_BVH_CWBVH ? "cwbvh" : "bvh2") << "|" << (q == RQ_ANY ? "any" : "closest") << "|"
       << cls;
    return os.str();
}

static bool cache_lookup(const char* path, const std::string& key, rq_launch* out) {
    if (!path) return false;
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        std::string k;
        rq_launch l{};
        if (is >> k >> l.block_size >> l.blocks_per_sm >> l.smem_stack >> l.postpone_ratio >> l.fetch_nd >> l.fetch_nw &&
            k == key) {
            *out = l;
            found = true;  // last entry wins
        }
    }
    return found;
}

static void cache_store(const char* path, const std::string& key, const rq_launch& l) {
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << key << " " << l.block_size << " " << l.blocks_per_sm << " " << l.smem_stack << " " << l.postpone_ratio << " "
      << l.fetch_nd << " " << l.fetch_nw << "\n";
}

// Second tuning stage: the refill thresholds (Nd, Nw; Nd -1 stands for 0)
// and, for CWBVH, the triangle postponing ratio, tried on the launch shape
// the first stage chose.
struct FetchChoice {
    int nd, nw;
};
constexpr FetchChoice kFetchChoices[] = {{2, 8}, {4, 4}, {1, 16}, {-1, 1}};
constexpr float kRatioChoices[] = {0.2f, 0.3f};

}  // namespace rq

extern "C" {

rq_status rq_autotune(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits, int64_t count,
                      rq_query query, const char* cache_path, rq_launch* out, void* stream) {
    if (!ctx || !scene || !rays || !hits || count <= 0 || !out) return RQ_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const std::string key = tune_key(scene->kind, query, count);
    if (cache_lookup(cache_path, key, out)) return RQ_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    RQ_CUDA(cudaEventCreate(&e0));
    RQ_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    rq_launch best = resolve_launch(scene->kind, query, nullptr);
    const int blocks[] = {64, 128, 256};
    const int stacks[] = {4, 8, 16};
    const float ratios[] = {0.2f, -1.0f};
    rq_status st = RQ_OK;
    for (int bs : blocks)
        for (int sm : stacks)
            for (float rt : ratios) {
                if (scene->kind == RQ_BVH_BVH2 && rt > 0.f) continue;  // no triangle postponing in BVH2
                rq_launch l{};
                l.block_size = bs;
                l.smem_stack = sm;
                l.postpone_ratio = rt;
                float ms_runs[3];
                for (int r = 0; r < 4 && st == RQ_OK; ++r) {
                    cudaEventRecord(e0, s);
                    st = rq_trace(ctx, scene, rays, hits, count, query, &l, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) ms_runs[r - 1] = ms;  // first run warms up
                }
                if (st != RQ_OK) break;
                std::sort(ms_runs, ms_runs + 3);
                if (ms_runs[1] < best_ms) {
                    best_ms = ms_runs[1];
                    best = resolve_launch(scene->kind, query, &l);
                    best.postpone_ratio = rt < 0.f ? -1.0f : rt;
                }
            }
    if (st == RQ_OK) {
        const rq_launch shape = best;
        for (const FetchChoice& fc : kFetchChoices)
            for (float rt : kRatioChoices) {
                if (st != RQ_OK) break;
                rq_launch l = shape;
                l.fetch_nd = fc.nd;
                l.fetch_nw = fc.nw;
                if (scene->kind == RQ_BVH_CWBVH && shape.postpone_ratio > 0.f) l.postpone_ratio = rt;
                else if (rt != kRatioChoices[0]) continue;  // the ratio does not apply
                float ms_runs[3];
                for (int r = 0; r < 4 && st == RQ_OK; ++r) {
                    cudaEventRecord(e0, s);
                    st = rq_trace(ctx, scene, rays, hits, count, query, &l, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) ms_runs[r - 1] = ms;
                }
                if (st != RQ_OK) break;
                std::sort(ms_runs, ms_runs + 3);
                if (ms_runs[1] < best_ms) {
                    best_ms = ms_runs[1];
                    best = l;
                }
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RQ_OK) return st;
    *out = best;
    cache_store(cache_path, key, best);
    return RQ_OK;
}

rq_status rq_autotune_batch(rq_ctx_t ctx, const rq_batch_item* items, int n_items, rq_query query,
                            const char* cache_path, rq_batch_params* out, void* stream) {
    if (!ctx || !items || n_items <= 0 || !out) return RQ_ERR_INVALID_ARG;
    int64_t total = 0, max_count = 0;
    for (int i = 0; i < n_items; ++i) {
        total += items[i].count;
        max_count = std::max(max_count, items[i].count);
    }
    std::string key;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        key = "batch|" + tune_key(items[0].scene->kind, query, total) + "|" + std::to_string(n_items);
        rq_launch l{};
        std::ifstream f(cache_path ? cache_path : "");
        std::string line;
        bool found = false;
        long long thr = -1;
        int graph = 0;
        while (cache_path && std::getline(f, line)) {
            std::istringstream is(line);
            std::string k;
            rq_launch c{};
            long long t;
            int g;
            if (is >> k >> c.block_size >> c.blocks_per_sm >> c.smem_stack >> c.postpone_ratio >> c.fetch_nd >>
                    c.fetch_nw >> t >> g &&
                k == key) {
                l = c;
                thr = t;
                graph = g;
                found = true;
            }
        }
        if (found) {
            out->launch = l;
            out->sort_threshold = thr;
            out->use_graph = graph;
            return RQ_OK;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaEvent_t e0, e1;
    RQ_CUDA(cudaEventCreate(&e0));
    RQ_CUDA(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    rq_batch_params best{};
    const int blocks[] = {64, 128, 256};
    const int stacks[] = {8, 16};
    // Sort thresholds: never, items of at least 1M rays, every item.
    const int64_t thresholds[] = {-1, std::min<int64_t>(max_count, 1 << 20), 0};
    rq_status st = RQ_OK;
    for (int64_t thr : thresholds)
        for (int bs : blocks)
            for (int sm : stacks) {
                rq_batch_params bp{};
                bp.launch.block_size = bs;
                bp.launch.smem_stack = sm;
                bp.sort_threshold = thr;
                bp.use_graph = s != nullptr;
                rq_batch_t b = nullptr;
                st = rq_batch_create(ctx, items, n_items, query, &bp, &b);
                if (st != RQ_OK) break;
                float ms_runs[2];
                for (int r = 0; r < 3 && st == RQ_OK; ++r) {
                    cudaEventRecord(e0, s);
                    st = rq_batch_run(b, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) ms_runs[r - 1] = ms;
                }
                rq_batch_destroy(b);
                if (st != RQ_OK) break;
                const float ms = std::min(ms_runs[0], ms_runs[1]);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = bp;
                }
            }
    if (st == RQ_OK) {
        // The first stage ran with the default refill thresholds and ratio:
        // write them out, so that a first-stage winner the second stage does
        // not beat is returned (and cached) as the explicit launch it ran.
        best.launch = resolve_launch(items[0].scene->kind, query, &best.launch);
        const rq_batch_params shape = best;
        const bool cw = items[0].scene->kind == RQ_BVH_CWBVH;
        for (const FetchChoice& fc : kFetchChoices)
            for (float rt : kRatioChoices) {
                if (st != RQ_OK) break;
                if (!cw && rt != kRatioChoices[0]) continue;  // no triangle postponing in BVH2
                rq_batch_params bp = shape;
                bp.launch.fetch_nd = fc.nd;
                bp.launch.fetch_nw = fc.nw;
                if (cw) bp.launch.postpone_ratio = rt;
                rq_batch_t b = nullptr;
                st = rq_batch_create(ctx, items, n_items, query, &bp, &b);
                if (st != RQ_OK) break;
                float ms_runs[2];
                for (int r = 0; r < 3 && st == RQ_OK; ++r) {
                    cudaEventRecord(e0, s);
                    st = rq_batch_run(b, s);
                    cudaEventRecord(e1, s);
                    cudaEventSynchronize(e1);
                    float ms = 0.f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (r > 0) ms_runs[r - 1] = ms;
                }
                rq_batch_destroy(b);
                if (st != RQ_OK) break;
                const float ms = std::min(ms_runs[0], ms_runs[1]);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = bp;
                }
            }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RQ_OK) return st;
    *out = best;
    if (cache_path) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        std::ofstream f(cache_path, std::ios::app);
        const rq_launch& l = best.launch;
        f << key << " " << l.block_size << " " << l.blocks_per_sm << " " << l.smem_stack << " " << l.postpone_ratio << " "
          << l.fetch_nd << " " << l.fetch_nw << " " << (long long)best.sort_threshold << " " << best.use_graph << "\n";
    }
    return RQ_OK;
}

}  // extern "C"
