// Converters from the builder's trees to the GPU layouts the trace kernels
// read.  The byte layouts, the depth-first emission order and the encodings are
// those of the reference converter (src/GPUBVHConverter.cpp:10-378), so a tree
// converted here and by the reference gives the same node bytes.  Deliberate
// differences, each guarding a reference edge case:
//   * Woop rows are computed in double precision and rounded once (the
//     reference inverts a float 4x4 matrix, src/WoopTriangleHelper.h:318-354),
//     so rows agree to a few ulp, not bitwise.
//   * a degenerate triangle gets all-zero rows, which no ray can hit (the
//     reference substitutes the identity matrix, a phantom unit triangle at the
//     origin, src/WoopTriangleHelper.h:345-346);
//   * V0.x = -0.0f is stored as +0.0f so it cannot collide with the BVH2 leaf
//     terminator bit pattern 0x80000000 (src/TraversalKernelBVH2.cu:132);
//   * an axis whose quantised upper bound would reach 256 (and wrap to 0 in the
//     reference's uint8 store, src/GPUBVHConverter.cpp:306-316) gets the next
//     larger exponent;
//   * a zero-extent axis gets exponent 0 (the reference converts -inf to char,
//     which is undefined; x86 yields 0), and exponents are clamped to int8.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "host_common.h"

namespace rq {

static inline float bits_to_float(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
static inline float int_bits(int32_t i) {
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}

// Woop transform (src/GPUBVHConverter.cpp:380-403).  With e0 = v0-v2, e1 =
// v1-v2, n = e0 x e1 (float, as the reference computes them) the affine map
// M = [e0 e1 n v2] takes the unit triangle to the triangle; the rows of M^-1
// give the triangle-space z (V0, with w negated), u (V1) and v (V2).
void woopify(const V3& v0, const V3& v1, const V3& v2, float out[12]) {
    const V3 e0 = v0 - v2, e1 = v1 - v2;
    const V3 n = cross(e0, e1);
    const double a[3][3] = {{e0.x, e1.x, n.x}, {e0.y, e1.y, n.y}, {e0.z, e1.z, n.z}};
    const double t[3] = {v2.x, v2.y, v2.z};
    // Adjugate / determinant of the 3x3 linear part.
    double c[3][3];
    c[0][0] = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    c[0][1] = a[0][2] * a[2][1] - a[0][1] * a[2][2];
    c[0][2] = a[0][1] * a[1][2] - a[0][2] * a[1][1];
    c[1][0] = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    c[1][1] = a[0][0] * a[2][2] - a[0][2] * a[2][0];
    c[1][2] = a[0][2] * a[1][0] - a[0][0] * a[1][2];
    c[2][0] = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    c[2][1] = a[0][1] * a[2][0] - a[0][0] * a[2][1];
    c[2][2] = a[0][0] * a[1][1] - a[0][1] * a[1][0];
    const double det = a[0][0] * c[0][0] + a[0][1] * c[1][0] + a[0][2] * c[2][0];
    if (det == 0.0 || !std::isfinite(det)) {
        for (int k = 0; k < 12; ++k) out[k] = 0.0f;
        return;
    }
    double inv[3][4];
    const double rdet = 1.0 / det;
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) inv[r][k] = c[r][k] * rdet;
        inv[r][3] = -(inv[r][0] * t[0] + inv[r][1] * t[1] + inv[r][2] * t[2]);
    }
    // V0 = (row 2, -w), V1 = row 0, V2 = row 1.
    out[0] = (float)inv[2][0];
    out[1] = (float)inv[2][1];
    out[2] = (float)inv[2][2];
    out[3] = (float)(-inv[2][3]);
    for (int k = 0; k < 4; ++k) out[4 + k] = (float)inv[0][k];
    for (int k = 0; k < 4; ++k) out[8 + k] = (float)inv[1][k];
    if (out[0] == 0.0f) out[0] = 0.0f;  // -0.0f would read as a BVH2 leaf terminator
}

static void append_triangle(const Mesh& m, int32_t prim, HostBVH& out) {
    const int32_t* tri = &m.i[3 * (int64_t)prim];
    float w[12];
    woopify(m.vert(tri[0]), m.vert(tri[1]), m.vert(tri[2]), w);
    out.woop.insert(out.woop.end(), w, w + 12);
    out.prim_index.push_back(prim);
    out.prim_index.push_back(-1);
    out.prim_index.push_back(-1);
}

// ---------------------------------------------------------------- BVH2 ----
// Node = 4 float4: (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y), (same for c1),
// (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z), (child0, child1 as int bits, 0, 0).
// A child >= 0 is the float4 index of an inner node; < 0 is ~(float4 index of
// the leaf's first Woop row).  (src/GPUBVHConverter.cpp:57-118)
void convert_bvh2(const Tree<2>& t, const Mesh& m, HostBVH& out) {
    out.kind = RQ_BVH_BVH2;
    out.nodes.clear();
    out.woop.clear();
    out.prim_index.clear();
    out.bounds = t.bounds;

    // Work list entries: a tree child code, its parent's node address and slot.
    struct Item { int32_t code; int32_t parent; int slot; };
    std::vector<Item> st;

    // A leaf-only scene gets an inner root over the leaf (box = everything) and
    // a never-hit leaf (inverted box), as the reference does
    // (src/GPUBVHConverter.cpp:21-38).
    TreeNode<2> synth{};
    const bool synth_root = t.root_is_leaf;
    std::vector<Leaf> leaves = t.leaves;
    std::vector<int32_t> refs = t.prim_refs;
    if (synth_root) {
        synth.count = 2;
        synth.child[0] = -2;
        int32_t first_prim = (t.leaves[0].count > 0) ? t.prim_refs[t.leaves[0].first] : -1;
        if (first_prim >= 0) {
            leaves.push_back(Leaf{(int32_t)refs.size(), 1});
            refs.push_back(first_prim);
            synth.child[1] = -(int32_t)(leaves.size() - 1) - 2;
        } else {
            leaves.push_back(Leaf{0, 0});
            synth.child[1] = -(int32_t)(leaves.size() - 1) - 2;
        }
        for (int a = 0; a < 3; ++a) {
            synth.lo[0][a] = -FLT_MAX; synth.hi[0][a] = FLT_MAX;
            synth.lo[1][a] = FLT_MAX;  synth.hi[1][a] = -FLT_MAX;
        }
    }
    auto node_of = [&](int32_t code) -> const TreeNode<2>& {
        return (synth_root && code == 0) ? synth : t.nodes[code];
    };

    st.push_back({0, -1, 0});
    int64_t n_nodes = 0, n_leaves = 0;
    while (!st.empty()) {
        const Item it = st.back();
        st.pop_back();
        int32_t addr;
        if (it.code >= 0) {
            const TreeNode<2>& nd = node_of(it.code);
            addr = (int32_t)(out.nodes.size() / 4);
            const float c[16] = {nd.lo[0][0], nd.hi[0][0], nd.lo[0][1], nd.hi[0][1],
                                 nd.lo[1][0], nd.hi[1][0], nd.lo[1][1], nd.hi[1][1],
                                 nd.lo[0][2], nd.hi[0][2], nd.lo[1][2], nd.hi[1][2],
                                 0.f, 0.f, 0.f, 0.f};
            out.nodes.insert(out.nodes.end(), c, c + 16);
            st.push_back({nd.child[0], addr, 0});
            st.push_back({nd.child[1], addr, 1});
            ++n_nodes;
        } else {
            const Leaf& lf = leaves[-it.code - 2];
            addr = ~(int32_t)(out.woop.size() / 4);
            for (int32_t k = 0; k < lf.count; ++k) append_triangle(m, refs[lf.first + k], out);
            const float term[4] = {bits_to_float(0x80000000u), 0.f, 0.f, 0.f};
            out.woop.insert(out.woop.end(), term, term + 4);
            out.prim_index.push_back(-1);
            ++n_leaves;
        }
        if (it.parent >= 0) out.nodes[(size_t)it.parent * 4 + 12 + it.slot] = int_bits(addr);
    }
    out.node_count = n_nodes;
    out.leaf_count = n_leaves;
}

// --------------------------------------------------------------- CWBVH ----
// Node = 5 float4 (80 B): n0 = (p.xyz, bytes{e.x, e.y, e.z, imask}),
// n1 = (child base node index, triangle base index, meta[0..3], meta[4..7]),
// n2..n4 = qlo.x[8] qlo.y[8] qlo.z[8] qhi.x[8] qhi.y[8] qhi.z[8] (uint8).
// (src/GPUBVHConverter.cpp:123-378)
namespace {

struct Child8 {
    int32_t code;
    float lo[3], hi[3];
};

// Greedy assignment of children to the 8 octant slots: repeatedly take the
// cheapest (slot, child) pair, cost = dot(child centre - node centre, slot
// direction), ties going to the lower slot, then the lower child; leftover
// (empty) children fill the free slots in order.  Same rule as the reference
// (src/GPUBVHConverter.cpp:170-260) so node bytes match.
void order_children(const float node_lo[3], const float node_hi[3], Child8 ch[8], const bool present[8],
                    Child8 out[8], bool out_present[8]) {
    float nc[3];
    for (int a = 0; a < 3; ++a) nc[a] = (node_lo[a] + node_hi[a]) * 0.5f;
    float cost[8][8];
    for (int s = 0; s < 8; ++s) {
        const float dx = (s & 4) ? -1.0f : 1.0f, dy = (s & 2) ? -1.0f : 1.0f, dz = (s & 1) ? -1.0f : 1.0f;
        for (int c = 0; c < 8; ++c) {
            if (!present[c]) {
                cost[s][c] = FLT_MAX;
                continue;
            }
            const float cx = (ch[c].lo[0] + ch[c].hi[0]) * 0.5f - nc[0];
            const float cy = (ch[c].lo[1] + ch[c].hi[1]) * 0.5f - nc[1];
            const float cz = (ch[c].lo[2] + ch[c].hi[2]) * 0.5f - nc[2];
            float d = cx * dx + cy * dy;
            d = d + cz * dz;
            cost[s][c] = d;
        }
    }
    int slot_of[8];
    bool slot_free[8];
    for (int k = 0; k < 8; ++k) { slot_of[k] = -1; slot_free[k] = true; }
    for (;;) {
        float best = FLT_MAX;
        int bs = -1, bc = -1;
        for (int s = 0; s < 8; ++s)
            for (int c = 0; c < 8; ++c)
                if (slot_of[c] < 0 && slot_free[s] && cost[s][c] < best) { best = cost[s][c]; bs = s; bc = c; }
        if (bs < 0) break;
        slot_free[bs] = false;
        slot_of[bc] = bs;
    }
    for (int c = 0; c < 8; ++c) {
        if (slot_of[c] >= 0) continue;
        for (int s = 0; s < 8; ++s)
            if (slot_free[s]) { slot_free[s] = false; slot_of[c] = s; break; }
    }
    for (int c = 0; c < 8; ++c) {
        out[slot_of[c]] = ch[c];
        out_present[slot_of[c]] = present[c];
    }
}

int8_t axis_exponent(float extent) {
    const float r = std::ceil(std::log2(extent / 255.0f));
    if (!std::isfinite(r)) return 0;
    return (int8_t)std::max(-127.0f, std::min(127.0f, r));
}

}  // namespace

// The converter's output order, restated so subtrees can be converted in
// parallel with identical bytes.  Sequentially, a node's processing appends
// its inner children's 80 B slots (one contiguous block, in slot order) and
// its leaf children's triangles (slot order), then pushes the inner children;
// the stack then converts them last slot first, each subtree completely
// before the next.  So every subtree owns one contiguous range of node slots
// and one of triangles, whose starts follow from the subtree sizes: the ranges
// are computed up front and the subtrees filled independently.
namespace {

template <class EmitPrim>
struct CwbvhWriter {
    const Tree<8>& t;
    EmitPrim& emit;            // emit(prim, triangle index)
    HostBVH& out;
    std::vector<int64_t> desc;  // inner descendants of each node
    std::vector<int64_t> tris;  // triangles below each node
    int64_t grain = 0;
    std::atomic<int> spare{0};

    CwbvhWriter(const Tree<8>& tree, EmitPrim& e, HostBVH& o) : t(tree), emit(e), out(o) {}

    void sizes() {
        const size_t n = t.nodes.size();
        desc.assign(n, 0);
        tris.assign(n, 0);
        std::vector<std::pair<int32_t, bool>> st{{0, false}};
        while (!st.empty()) {
            auto [v, done] = st.back();
            st.pop_back();
            const TreeNode<8>& nd = t.nodes[v];
            if (!done) {
                st.push_back({v, true});
                for (int c = 0; c < 8; ++c)
                    if (nd.child[c] >= 0) st.push_back({nd.child[c], false});
                continue;
            }
            for (int c = 0; c < 8; ++c) {
                const int32_t code = nd.child[c];
                if (code >= 0) {
                    desc[v] += 1 + desc[code];
                    tris[v] += tris[code];
                } else if (code <= -2) {
                    tris[v] += t.leaves[-code - 2].count;
                }
            }
        }
    }

    // Converts node v, whose slot is at float4 `addr`, with its children's
    // block at float4 `node_cur` and its triangles from `tri_cur` on.
    void convert(int32_t v, int64_t addr, int64_t node_cur, int64_t tri_cur) {
        const TreeNode<8>& nd = t.nodes[v];
        Child8 ch[8];
        bool present[8];
        float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (int c = 0; c < 8; ++c) {
            present[c] = nd.child[c] != -1;
            ch[c].code = nd.child[c];
            for (int a = 0; a < 3; ++a) { ch[c].lo[a] = nd.lo[c][a]; ch[c].hi[a] = nd.hi[c][a]; }
            if (!present[c]) continue;
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::fmin(lo[a], nd.lo[c][a]);
                hi[a] = std::fmax(hi[a], nd.hi[c][a]);
            }
        }
        Child8 oc[8];
        bool op[8];
        order_children(lo, hi, ch, present, oc, op);

        // Per-axis exponent; grow it while some child's upper bound would not fit in a byte.
        int8_t e[3];
        for (int a = 0; a < 3; ++a) {
            e[a] = axis_exponent(hi[a] - lo[a]);
            for (;;) {
                const float scale = std::ldexp(1.0f, e[a]);  // = powf(2, e), exactly
                bool fits = true;
                for (int c = 0; c < 8; ++c)
                    if (op[c] && (int)std::ceil((oc[c].hi[a] - lo[a]) / scale) > 255) fits = false;
                if (fits || e[a] >= 127) break;
                ++e[a];
            }
        }

        uint8_t* node_bytes = reinterpret_cast<uint8_t*>(&out.nodes[(size_t)addr * 4]);
        uint8_t imask = 0;
        int64_t inner = 0, leaf_tris = 0;
        int64_t child_addr[8];
        for (int c = 0; c < 8; ++c) {
            child_addr[c] = -1;
            if (!op[c]) continue;
            for (int a = 0; a < 3; ++a) {
                const float scale = std::ldexp(1.0f, e[a]);
                node_bytes[32 + c + 8 * a] = (uint8_t)(int)std::floor((oc[c].lo[a] - lo[a]) / scale);
                node_bytes[32 + c + 8 * (3 + a)] = (uint8_t)(int)std::ceil((oc[c].hi[a] - lo[a]) / scale);
            }
            uint8_t meta;
            if (oc[c].code >= 0) {
                child_addr[c] = node_cur + 5 * inner;
                imask |= (uint8_t)(1u << c);
                meta = (uint8_t)((1u << 5) | ((24u + c) & 31u));
                ++inner;
            } else {
                const Leaf& lf = t.leaves[-oc[c].code - 2];
                const uint32_t unary = lf.count == 1 ? 1u : (lf.count == 2 ? 3u : 7u);
                meta = (uint8_t)((unary << 5) | ((uint32_t)leaf_tris & 31u));
                for (int32_t k = 0; k < lf.count; ++k) emit(t.prim_refs[lf.first + k], tri_cur + leaf_tris + k);
                leaf_tris += lf.count;
            }
            node_bytes[24 + c] = meta;
        }
        float* n = &out.nodes[(size_t)addr * 4];
        n[0] = lo[0];
        n[1] = lo[1];
        n[2] = lo[2];
        uint8_t* w = reinterpret_cast<uint8_t*>(&n[3]);
        w[0] = (uint8_t)e[0];
        w[1] = (uint8_t)e[1];
        w[2] = (uint8_t)e[2];
        w[3] = imask;
        n[4] = int_bits(inner ? (int32_t)(node_cur / 5) : 0);
        n[5] = int_bits(leaf_tris ? (int32_t)tri_cur : 0);

        // Subtrees, last slot first, each in its own ranges.
        int64_t nc = node_cur + 5 * inner, tc = tri_cur + leaf_tris;
        std::vector<std::thread> helpers;
        for (int c = 7; c >= 0; --c) {
            if (child_addr[c] < 0) continue;
            const int32_t code = oc[c].code;
            if (tris[code] >= grain && spare.fetch_sub(1) > 0) {
                helpers.emplace_back([this, code, a = child_addr[c], nc, tc] { convert(code, a, nc, tc); });
            } else {
                if (tris[code] >= grain) spare.fetch_add(1);
                convert(code, child_addr[c], nc, tc);
            }
            nc += 5 * desc[code];
            tc += tris[code];
        }
        for (auto& h : helpers) {
            h.join();
            spare.fetch_add(1);
        }
    }
};

}  // namespace

template <class EmitPrim>
static void convert_cwbvh_impl(const Tree<8>& t, EmitPrim&& emit, HostBVH& out, int threads) {
    out.kind = RQ_BVH_CWBVH;
    out.bounds = t.bounds;
    CwbvhWriter<EmitPrim> wr(t, emit, out);
    wr.sizes();
    const int64_t n_nodes = 1 + wr.desc[0], n_tris = wr.tris[0];
    out.nodes.assign((size_t)n_nodes * 20, 0.0f);
    out.woop.assign((size_t)n_tris * 12, 0.0f);
    out.prim_index.assign((size_t)n_tris * 3, 0);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    wr.spare = threads - 1;
    wr.grain = threads > 1 ? std::max<int64_t>(4096, n_tris / (8 * (int64_t)threads)) : INT64_MAX;
    wr.convert(0, 0, 5, 0);
    int64_t n_leaves = 0;
    for (const TreeNode<8>& nd : t.nodes)
        for (int c = 0; c < 8; ++c) n_leaves += nd.child[c] <= -2;
    out.node_count = n_nodes;
    out.leaf_count = n_leaves;
}

void convert_cwbvh(const Tree<8>& t, const Mesh& m, HostBVH& out, int threads) {
    auto emit = [&](int32_t prim, int64_t k) {
        const int32_t* tri = &m.i[3 * (int64_t)prim];
        woopify(m.vert(tri[0]), m.vert(tri[1]), m.vert(tri[2]), &out.woop[(size_t)k * 12]);
        out.prim_index[(size_t)k * 3] = prim;
        out.prim_index[(size_t)k * 3 + 1] = -1;
        out.prim_index[(size_t)k * 3 + 2] = -1;
    };
    convert_cwbvh_impl(t, emit, out, threads);
}

void convert_cwbvh_instances(const Tree<8>& t, const float* rows12, const int32_t* extra, HostBVH& out,
                             int threads) {
    auto emit = [&](int32_t k, int64_t slot) {
        std::copy(rows12 + 12 * (int64_t)k, rows12 + 12 * (int64_t)k + 12, &out.woop[(size_t)slot * 12]);
        out.prim_index[(size_t)slot * 3] = k;
        out.prim_index[(size_t)slot * 3 + 1] = extra[k];
        out.prim_index[(size_t)slot * 3 + 2] = -1;
    };
    convert_cwbvh_impl(t, emit, out, threads);
}

}  // namespace rq
