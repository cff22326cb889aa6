// Host-side shared types of librq: vectors, seeded hashing RNG, the BVH trees
// produced by the builder and the converted (GPU-layout) buffers.
#pragma once

#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <vector>

#include "../../include/rq.h"

namespace rq {

struct V3 {
    float x, y, z;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 vmin(V3 a, V3 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y), std::fmin(a.z, b.z)}; }
inline V3 vmax(V3 a, V3 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)}; }
inline float comp(const V3& a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct Box {
    V3 lo{INFINITY, INFINITY, INFINITY};
    V3 hi{-INFINITY, -INFINITY, -INFINITY};
    void grow(const V3& p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void grow(const Box& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    float area() const {
        float dx = hi.x - lo.x, dy = hi.y - lo.y, dz = hi.z - lo.z;
        if (!(dx >= 0.f && dy >= 0.f && dz >= 0.f)) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

// Stateless 64-bit hash (splitmix64 finaliser); every generated quantity is
// hash(seed, stream, index) so generation is order- and thread-independent.
inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
inline uint64_t hash3(uint64_t seed, uint64_t stream, uint64_t i) {
    return mix64(mix64(seed ^ mix64(stream * 0x632BE59BD9B4E019ull)) + i);
}
// Uniform float in [0,1) with 24 random bits.
inline float u01(uint64_t seed, uint64_t stream, uint64_t i) {
    return (float)(hash3(seed, stream, i) >> 40) * (1.0f / 16777216.0f);
}

// Runs fn(0 .. n-1) on up to `threads` host threads (0: all cores); each
// index runs once, in no particular order.
inline void parallel_tasks(int64_t n, int threads, const std::function<void(int64_t)>& fn) {
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const int workers = (int)std::min<int64_t>(n, threads);
    if (workers <= 1) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<int64_t> next{0};
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w)
        pool.emplace_back([&] {
            for (int64_t i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
        });
    for (auto& th : pool) th.join();
}

struct Mesh {
    std::vector<float> v;    // 3 per vertex
    std::vector<int32_t> i;  // 3 per triangle
    int64_t nv() const { return (int64_t)v.size() / 3; }
    int64_t nt() const { return (int64_t)i.size() / 3; }
    V3 vert(int64_t k) const { return {v[3 * k], v[3 * k + 1], v[3 * k + 2]}; }
};

// Pre-conversion tree, one record per node.  child[k] >= 0 is an inner node,
// child[k] <= -2 is leaf (-child-2), -1 is an empty slot.  Children occupy
// slots 0..count-1, as the reference's BVHNNode<N> (src/EmbreeBVHBuilder.h:7-37).
template <int W>
struct TreeNode {
    int32_t child[W];
    float lo[W][3];
    float hi[W][3];
    int count;
};

struct Leaf {
    int32_t first;  // into Tree::prim_refs
    int32_t count;
};

template <int W>
struct Tree {
    std::vector<TreeNode<W>> nodes;  // node 0 is the root
    std::vector<Leaf> leaves;
    std::vector<int32_t> prim_refs;
    bool root_is_leaf = false;       // the whole scene is one leaf (leaves[0])
    Box bounds;
};

// Converted GPU-layout buffers (the output of the reference's converters,
// GPUBVHIntermediates, src/GPUBVHConverter.h:6-11).
struct HostBVH {
    rq_bvh_kind kind;
    std::vector<float> nodes;        // float4 units
    std::vector<float> woop;         // float4 units
    std::vector<int32_t> prim_index; // one per Woop float4
    int64_t node_count = 0;
    int64_t leaf_count = 0;
    int depth = 0;
    Box bounds;
    // The pre-conversion tree is kept for converter cross-checks (absent
    // when the buffers were loaded from a scene file).
    Tree<2> tree2;
    Tree<8> tree8;
    bool has_tree = true;
};

// Builders (builder.cpp)
// max_frags > 1: pre-split badly fitting triangles into up to max_frags
// references with clipped bounds (power of two).  split_budget > 0: spatial
// splits during the build, adding at most split_budget * triangles
// duplicate references.
void build_bvh2_tree(const Mesh& m, int max_leaf, int bins, int max_depth, bool big_leaves, int threads,
                     Tree<2>& out, int max_frags = 1, float split_budget = 0.f);
// Binary tree over axis-aligned boxes (lo xyz, hi xyz per box; box k is
// primitive k), e.g. the world bounds of instances for a top-level tree.
void build_bvh2_tree_boxes(const float* boxes, int64_t n, int bins, int max_depth, int threads, Tree<2>& out);
// SAH treelet restructuring of a binary tree (7-leaf treelets, `passes`
// bottom-up sweeps); leaves and their primitives are unchanged.
void treelet_optimize(Tree<2>& t, int passes, int threads);
void collapse_to_bvh8(const Tree<2>& t2, Tree<8>& out, int threads = 1);
int tree_depth2(const Tree<2>& t);
int tree_depth8(const Tree<8>& t);

// Converters (convert.cpp)
void woopify(const V3& v0, const V3& v1, const V3& v2, float out[12]);
void convert_bvh2(const Tree<2>& t, const Mesh& m, HostBVH& out);
void convert_cwbvh(const Tree<8>& t, const Mesh& m, HostBVH& out, int threads = 1);
// CWBVH nodes over a tree of instances: each leaf primitive k is emitted as
// the 3 rows of rows12[12 k ..] (the instance's world-to-object transform) in
// place of Woop rows, with primitive-map entries (k, extra[k], -1).
void convert_cwbvh_instances(const Tree<8>& t, const float* rows12, const int32_t* extra, HostBVH& out,
                             int threads = 1);

// Scene generators (scenegen.cpp)
void gen_heightfield_boxes(uint64_t seed, int grid, int n_boxes, float bmin, float bmax, Mesh& m);
void gen_city(uint64_t seed, int n_buildings, Mesh& m);
void gen_spheres_terrain(uint64_t seed, int64_t target_tris, Mesh& m);

}  // namespace rq

// Opaque handle of the C ABI's host-side BVH (rq_host_bvh_t).
struct rq_host_bvh {
    rq::HostBVH b;
};
