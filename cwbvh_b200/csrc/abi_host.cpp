// Host-only entry points of the C ABI: BVH build + conversion, the Woop
// transform, procedural scenes and status strings.  Nothing here touches the
// GPU, so these calls work on a machine without one.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <new>

#include "host_common.h"

// SAH treelet passes over the binary tree of a CWBVH build when the caller
// asks for the default.
#ifndef RQ_DEFAULT_TREELET_PASSES
#define RQ_DEFAULT_TREELET_PASSES 4
#endif
// Spatial-split budget (duplicate references, percent of the triangles) when
// the caller asks for the default.
#ifndef RQ_DEFAULT_SPATIAL_SPLITS
#define RQ_DEFAULT_SPATIAL_SPLITS 200
#endif

using namespace rq;


template <int W>
static void export_tree(const Tree<W>& t, int32_t* codes, float* boxes, int32_t* lf, int32_t* lc, int32_t* refs) {
    for (size_t n = 0; n < t.nodes.size(); ++n) {
        for (int c = 0; c < W; ++c) {
            if (codes) codes[n * W + c] = t.nodes[n].child[c];
            if (boxes)
                for (int a = 0; a < 3; ++a) {
                    boxes[(n * W + c) * 6 + a] = t.nodes[n].lo[c][a];
                    boxes[(n * W + c) * 6 + 3 + a] = t.nodes[n].hi[c][a];
                }
        }
    }
    for (size_t l = 0; l < t.leaves.size(); ++l) {
        if (lf) lf[l] = t.leaves[l].first;
        if (lc) lc[l] = t.leaves[l].count;
    }
    if (refs) std::copy(t.prim_refs.begin(), t.prim_refs.end(), refs);
}

extern "C" {

const char* rq_status_string(rq_status s) {
    switch (s) {
        case RQ_OK: return "RQ_OK";
        case RQ_ERR_INVALID_ARG: return "RQ_ERR_INVALID_ARG";
        case RQ_ERR_OOM: return "RQ_ERR_OOM";
        case RQ_ERR_STACK_OVERFLOW: return "RQ_ERR_STACK_OVERFLOW";
        case RQ_ERR_TIMEOUT: return "RQ_ERR_TIMEOUT";
        case RQ_ERR_CUDA: return "RQ_ERR_CUDA";
        case RQ_ERR_BAD_SCENE: return "RQ_ERR_BAD_SCENE";
        case RQ_ERR_NOT_FOUND: return "RQ_ERR_NOT_FOUND";
        case RQ_ERR_BUDGET: return "RQ_ERR_BUDGET";
        case RQ_ERR_CANCELLED: return "RQ_ERR_CANCELLED";
        case RQ_ERR_NO_DEVICE: return "RQ_ERR_NO_DEVICE";
    }
    return "RQ_ERR_UNKNOWN";
}

rq_status rq_build_bvh(const float* vertices, int64_t nv, const int32_t* indices, int64_t nt, rq_bvh_kind kind,
                       const rq_build_params* params, rq_host_bvh_t* out) {
    if (!out || nv < 0 || nt < 0 || (nv > 0 && !vertices) || (nt > 0 && !indices)) return RQ_ERR_INVALID_ARG;
    if (kind != RQ_BVH_CWBVH && kind != RQ_BVH_BVH2) return RQ_ERR_INVALID_ARG;
    if (nt > (int64_t)INT32_MAX / 3) return RQ_ERR_INVALID_ARG;
    for (int64_t k = 0; k < 3 * nt; ++k)
        if (indices[k] < 0 || indices[k] >= nv) return RQ_ERR_INVALID_ARG;
    rq_build_params bp{4, 32, 30, 0, 1, RQ_DEFAULT_TREELET_PASSES, RQ_DEFAULT_SPATIAL_SPLITS};
    if (params) {
        if (params->max_leaf_size > 0) bp.max_leaf_size = params->max_leaf_size;
        if (params->sah_bins > 0) bp.sah_bins = params->sah_bins;
        if (params->max_depth > 0) bp.max_depth = params->max_depth;
        bp.threads = params->threads;
        if (params->presplit > 0) bp.presplit = params->presplit;
        if (params->treelet_passes != 0) bp.treelet_passes = std::max(0, params->treelet_passes);
        if (params->spatial_splits != 0) bp.spatial_splits = std::max(0, params->spatial_splits);
    }
    if (bp.presplit != 1 && bp.presplit != 2 && bp.presplit != 4 && bp.presplit != 8) return RQ_ERR_INVALID_ARG;
    if (bp.spatial_splits > 400) return RQ_ERR_INVALID_ARG;
    const float split_budget = 0.01f * (float)bp.spatial_splits;
    rq_host_bvh* h = new (std::nothrow) rq_host_bvh();
    if (!h) return RQ_ERR_OOM;
    try {
        Mesh m;
        m.v.assign(vertices, vertices + 3 * nv);
        m.i.assign(indices, indices + 3 * nt);
        h->b.kind = kind;
        if (kind == RQ_BVH_BVH2) {
            build_bvh2_tree(m, std::max(1, bp.max_leaf_size), bp.sah_bins, bp.max_depth, true, bp.threads, h->b.tree2,
                            bp.presplit, split_budget);
            if (bp.treelet_passes > 0 && !h->b.tree2.root_is_leaf) {
                // Restructuring may deepen the tree: keep it only within the
                // depth limit (stacks of BVH2 kernels are sized by it).
                Tree<2> plain = h->b.tree2;
                treelet_optimize(h->b.tree2, bp.treelet_passes, bp.threads);
                if (tree_depth2(h->b.tree2) > std::max(tree_depth2(plain), bp.max_depth + 1))
                    h->b.tree2 = std::move(plain);
            }
            convert_bvh2(h->b.tree2, m, h->b);
            h->b.depth = tree_depth2(h->b.tree2);
        } else {
            // The 8-wide tree's leaves hold at most 3 triangles (3 meta bits).
            const auto t0 = std::chrono::steady_clock::now();
            build_bvh2_tree(m, 3, bp.sah_bins, 48, false, bp.threads, h->b.tree2, bp.presplit, split_budget);
            const auto t1a = std::chrono::steady_clock::now();
            treelet_optimize(h->b.tree2, bp.treelet_passes, bp.threads);
            const auto t1 = std::chrono::steady_clock::now();
            collapse_to_bvh8(h->b.tree2, h->b.tree8, bp.threads);
            const auto t2 = std::chrono::steady_clock::now();
            convert_cwbvh(h->b.tree8, m, h->b, bp.threads);
            const auto t3 = std::chrono::steady_clock::now();
            h->b.depth = tree_depth8(h->b.tree8);
            if (std::getenv("RQ_LOG")) {
                auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
                std::fprintf(stderr, "rq_build_bvh: %lld tris, binary SAH %.1f ms, %d treelet passes %.1f ms, "
                             "8-wide collapse %.1f ms, CWBVH conversion %.1f ms\n", (long long)nt, ms(t0, t1a),
                             bp.treelet_passes, ms(t1a, t1), ms(t1, t2), ms(t2, t3));
            }
        }
    } catch (const std::bad_alloc&) {
        delete h;
        return RQ_ERR_OOM;
    }
    *out = h;
    return RQ_OK;
}

rq_status rq_host_bvh_info(rq_host_bvh_t bvh, rq_bvh_info* out) {
    if (!bvh || !out) return RQ_ERR_INVALID_ARG;
    const HostBVH& b = bvh->b;
    out->node_float4s = (int64_t)b.nodes.size() / 4;
    out->woop_float4s = (int64_t)b.woop.size() / 4;
    out->prim_index_count = (int64_t)b.prim_index.size();
    out->node_count = b.node_count;
    out->leaf_count = b.leaf_count;
    out->depth = b.depth;
    out->kind = b.kind;
    out->bounds_lo[0] = b.bounds.lo.x; out->bounds_lo[1] = b.bounds.lo.y; out->bounds_lo[2] = b.bounds.lo.z;
    out->bounds_hi[0] = b.bounds.hi.x; out->bounds_hi[1] = b.bounds.hi.y; out->bounds_hi[2] = b.bounds.hi.z;
    return RQ_OK;
}

rq_status rq_host_bvh_buffers(rq_host_bvh_t bvh, const float** nodes, const float** woop, const int32_t** prim_index) {
    if (!bvh) return RQ_ERR_INVALID_ARG;
    if (nodes) *nodes = bvh->b.nodes.data();
    if (woop) *woop = bvh->b.woop.data();
    if (prim_index) *prim_index = bvh->b.prim_index.data();
    return RQ_OK;
}

void rq_host_bvh_free(rq_host_bvh_t bvh) { delete bvh; }

rq_status rq_host_bvh_tree(rq_host_bvh_t bvh, int32_t* width, int64_t* n_nodes, int64_t* n_leaves,
                           int64_t* n_prim_refs, int32_t* root_is_leaf, int32_t* child_codes, float* child_boxes,
                           int32_t* leaf_first, int32_t* leaf_count, int32_t* prim_refs) {
    if (!bvh) return RQ_ERR_INVALID_ARG;
    const HostBVH& b = bvh->b;
    if (!b.has_tree) return RQ_ERR_NOT_FOUND;  // loaded from a scene file: buffers only
    if (b.kind == RQ_BVH_BVH2) {
        if (width) *width = 2;
        if (n_nodes) *n_nodes = (int64_t)b.tree2.nodes.size();
        if (n_leaves) *n_leaves = (int64_t)b.tree2.leaves.size();
        if (n_prim_refs) *n_prim_refs = (int64_t)b.tree2.prim_refs.size();
        if (root_is_leaf) *root_is_leaf = b.tree2.root_is_leaf ? 1 : 0;
        export_tree(b.tree2, child_codes, child_boxes, leaf_first, leaf_count, prim_refs);
    } else {
        if (width) *width = 8;
        if (n_nodes) *n_nodes = (int64_t)b.tree8.nodes.size();
        if (n_leaves) *n_leaves = (int64_t)b.tree8.leaves.size();
        if (n_prim_refs) *n_prim_refs = (int64_t)b.tree8.prim_refs.size();
        if (root_is_leaf) *root_is_leaf = 0;
        export_tree(b.tree8, child_codes, child_boxes, leaf_first, leaf_count, prim_refs);
    }
    return RQ_OK;
}

}  // extern "C"

template <int W>
static bool import_tree(int64_t n_nodes, const int32_t* codes, const float* boxes, int64_t n_leaves,
                        const int32_t* lf, const int32_t* lc, int64_t n_refs, const int32_t* refs, bool root_is_leaf,
                        int64_t nt, Tree<W>& t) {
    t = Tree<W>();
    t.root_is_leaf = root_is_leaf;
    t.prim_refs.assign(refs, refs + n_refs);
    for (int64_t l = 0; l < n_leaves; ++l) {
        if (lf[l] < 0 || lc[l] < 0 || (int64_t)lf[l] + lc[l] > n_refs) return false;
        if (W == 8 && (lc[l] < 1 || lc[l] > 3)) return false;
        t.leaves.push_back(Leaf{lf[l], lc[l]});
    }
    for (int32_t r : t.prim_refs)
        if (r < 0 || r >= nt) return false;
    for (int64_t n = 0; n < n_nodes; ++n) {
        TreeNode<W> nd{};
        int count = 0;
        for (int c = 0; c < W; ++c) {
            const int32_t code = codes[n * W + c];
            if (code >= n_nodes || (code <= -2 && -code - 2 >= n_leaves)) return false;
            if (code != -1 && c != count) return false;  // children occupy slots 0..count-1
            nd.child[c] = code;
            if (code != -1) ++count;
            for (int a = 0; a < 3; ++a) {
                nd.lo[c][a] = boxes[(n * W + c) * 6 + a];
                nd.hi[c][a] = boxes[(n * W + c) * 6 + 3 + a];
            }
        }
        nd.count = count;
        t.nodes.push_back(nd);
    }
    if (root_is_leaf && n_leaves < 1) return false;
    if (!root_is_leaf && n_nodes < 1) return false;
    // A tree: the root is nobody's child and every other node has one parent,
    // so the converters' depth-first walks end.
    std::vector<uint8_t> parents(t.nodes.size(), 0);
    for (const auto& nd : t.nodes)
        for (int c = 0; c < W; ++c)
            if (nd.child[c] >= 0 && ++parents[nd.child[c]] > 1) return false;
    if (!t.nodes.empty() && parents[0] != 0) return false;
    Box b;
    for (const auto& nd : t.nodes)
        for (int c = 0; c < nd.count; ++c) {
            b.grow(v3(nd.lo[c][0], nd.lo[c][1], nd.lo[c][2]));
            b.grow(v3(nd.hi[c][0], nd.hi[c][1], nd.hi[c][2]));
        }
    t.bounds = b;
    return true;
}

extern "C" {

rq_status rq_convert_tree(int32_t width, int64_t n_nodes, const int32_t* child_codes, const float* child_boxes,
                          int64_t n_leaves, const int32_t* leaf_first, const int32_t* leaf_count, int64_t n_prim_refs,
                          const int32_t* prim_refs, int32_t root_is_leaf, const float* vertices, int64_t nv,
                          const int32_t* indices, int64_t nt, rq_host_bvh_t* out) {
    if (!out || (width != 2 && width != 8) || n_nodes < 0 || n_leaves < 0 || n_prim_refs < 0 || nv < 0 || nt < 0)
        return RQ_ERR_INVALID_ARG;
    if ((n_nodes > 0 && (!child_codes || !child_boxes)) || (n_leaves > 0 && (!leaf_first || !leaf_count)) ||
        (n_prim_refs > 0 && !prim_refs) || (nt > 0 && (!indices || !vertices)))
        return RQ_ERR_INVALID_ARG;
    if (width == 8 && root_is_leaf) return RQ_ERR_INVALID_ARG;  // the CWBVH root is an inner node
    for (int64_t k = 0; k < 3 * nt; ++k)
        if (indices[k] < 0 || indices[k] >= nv) return RQ_ERR_INVALID_ARG;
    rq_host_bvh* h = new (std::nothrow) rq_host_bvh();
    if (!h) return RQ_ERR_OOM;
    try {
        Mesh m;
        m.v.assign(vertices, vertices + 3 * nv);
        m.i.assign(indices, indices + 3 * nt);
        bool ok;
        if (width == 2) {
            h->b.kind = RQ_BVH_BVH2;
            ok = import_tree<2>(n_nodes, child_codes, child_boxes, n_leaves, leaf_first, leaf_count, n_prim_refs,
                                prim_refs, root_is_leaf != 0, nt, h->b.tree2);
            if (ok) {
                convert_bvh2(h->b.tree2, m, h->b);
                h->b.depth = tree_depth2(h->b.tree2);
            }
        } else {
            h->b.kind = RQ_BVH_CWBVH;
            ok = import_tree<8>(n_nodes, child_codes, child_boxes, n_leaves, leaf_first, leaf_count, n_prim_refs,
                                prim_refs, false, nt, h->b.tree8);
            if (ok) {
                convert_cwbvh(h->b.tree8, m, h->b);
                h->b.depth = tree_depth8(h->b.tree8);
            }
        }
        if (!ok) {
            delete h;
            return RQ_ERR_INVALID_ARG;
        }
    } catch (const std::bad_alloc&) {
        delete h;
        return RQ_ERR_OOM;
    }
    *out = h;
    return RQ_OK;
}

rq_status rq_woopify(const float v0[3], const float v1[3], const float v2[3], float out_rows[12]) {
    if (!v0 || !v1 || !v2 || !out_rows) return RQ_ERR_INVALID_ARG;
    woopify(v3(v0[0], v0[1], v0[2]), v3(v1[0], v1[1], v1[2]), v3(v2[0], v2[1], v2[2]), out_rows);
    return RQ_OK;
}

static rq_status export_mesh(const Mesh& m, float** vertices, int64_t* nv, int32_t** indices, int64_t* nt) {
    float* v = (float*)std::malloc(sizeof(float) * std::max<size_t>(1, m.v.size()));
    int32_t* i = (int32_t*)std::malloc(sizeof(int32_t) * std::max<size_t>(1, m.i.size()));
    if (!v || !i) {
        std::free(v);
        std::free(i);
        return RQ_ERR_OOM;
    }
    std::copy(m.v.begin(), m.v.end(), v);
    std::copy(m.i.begin(), m.i.end(), i);
    *vertices = v;
    *indices = i;
    *nv = m.nv();
    *nt = m.nt();
    return RQ_OK;
}

rq_status rq_gen_heightfield_boxes(uint64_t seed, int grid, int n_boxes, float box_min, float box_max,
                                   float** vertices, int64_t* nv, int32_t** indices, int64_t* nt) {
    if (!vertices || !nv || !indices || !nt || grid < 1 || n_boxes < 0 || !(box_min >= 0.f) || box_max < box_min)
        return RQ_ERR_INVALID_ARG;
    try {
        Mesh m;
        gen_heightfield_boxes(seed, grid, n_boxes, box_min, box_max, m);
        return export_mesh(m, vertices, nv, indices, nt);
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}

rq_status rq_gen_city(uint64_t seed, int n_buildings, float** vertices, int64_t* nv, int32_t** indices, int64_t* nt) {
    if (!vertices || !nv || !indices || !nt || n_buildings < 1) return RQ_ERR_INVALID_ARG;
    try {
        Mesh m;
        gen_city(seed, n_buildings, m);
        return export_mesh(m, vertices, nv, indices, nt);
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}

rq_status rq_gen_spheres_terrain(uint64_t seed, int64_t target_tris, float** vertices, int64_t* nv, int32_t** indices,
                                 int64_t* nt) {
    if (!vertices || !nv || !indices || !nt || target_tris < 16) return RQ_ERR_INVALID_ARG;
    try {
        Mesh m;
        gen_spheres_terrain(seed, target_tris, m);
        return export_mesh(m, vertices, nv, indices, nt);
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}

void rq_free_mesh(float* vertices, int32_t* indices) {
    std::free(vertices);
    std::free(indices);
}

}  // extern "C"
