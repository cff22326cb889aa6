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

template <class EmitPrim>
static void convert_cwbvh_impl(const Tree<8>& t, EmitPrim&& emit, HostBVH& out);

void convert_cwbvh(const Tree<8>& t, const Mesh& m, HostBVH& out) {
    convert_cwbvh_impl(t, [&](int32_t prim) { append_triangle(m, prim, out); }, out);
}

void convert_cwbvh_instances(const Tree<8>& t, const float* rows12, const int32_t* extra, HostBVH& out) {
    convert_cwbvh_impl(t, [&](int32_t k) {
        out.woop.insert(out.woop.end(), rows12 + 12 * (int64_t)k, rows12 + 12 * (int64_t)k + 12);
        out.prim_index.push_back(k);
        out.prim_index.push_back(extra[k]);
        out.prim_index.push_back(-1);
    }, out);
}

template <class EmitPrim>
static void convert_cwbvh_impl(const Tree<8>& t, EmitPrim&& emit, HostBVH& out) {
    out.kind = RQ_BVH_CWBVH;
    out.nodes.assign(20, 0.0f);  // root slot
    out.woop.clear();
    out.prim_index.clear();
    out.bounds = t.bounds;

    struct Item { int32_t node; int32_t addr; };  // addr in float4 units
    std::vector<Item> st{{0, 0}};
    int64_t n_nodes = 0, n_leaves = 0;
    while (!st.empty()) {
        const Item it = st.back();
        st.pop_back();
        const TreeNode<8>& nd = t.nodes[it.node];
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

        uint8_t* node_bytes = reinterpret_cast<uint8_t*>(&out.nodes[(size_t)it.addr * 4]);
        uint8_t imask = 0;
        int32_t child_base = 0, tri_base = 0;
        int inner = 0, leaf_tris = 0;
        for (int c = 0; c < 8; ++c) {
            if (!op[c]) continue;
            uint8_t q[6];
            for (int a = 0; a < 3; ++a) {
                const float scale = std::ldexp(1.0f, e[a]);  // = powf(2, e), exactly
                q[a] = (uint8_t)(int)std::floor((oc[c].lo[a] - lo[a]) / scale);
                q[3 + a] = (uint8_t)(int)std::ceil((oc[c].hi[a] - lo[a]) / scale);
            }
            // The node buffer may grow below, so address it afresh each time.
            node_bytes = reinterpret_cast<uint8_t*>(&out.nodes[(size_t)it.addr * 4]);
            for (int k = 0; k < 6; ++k) node_bytes[32 + c + 8 * k] = q[k];
            uint8_t meta;
            if (oc[c].code >= 0) {
                const int32_t child_addr = (int32_t)(out.nodes.size() / 4);
                if (inner == 0) child_base = child_addr / 5;
                out.nodes.resize(out.nodes.size() + 20, 0.0f);
                imask |= (uint8_t)(1u << c);
                meta = (uint8_t)((1u << 5) | ((24u + c) & 31u));
                ++inner;
                st.push_back({oc[c].code, child_addr});
            } else {
                const Leaf& lf = t.leaves[-oc[c].code - 2];
                if (leaf_tris == 0) tri_base = (int32_t)(out.woop.size() / 12);
                const uint32_t unary = lf.count == 1 ? 1u : (lf.count == 2 ? 3u : 7u);
                meta = (uint8_t)((unary << 5) | ((uint32_t)leaf_tris & 31u));
                leaf_tris += lf.count;
                for (int32_t k = 0; k < lf.count; ++k) emit(t.prim_refs[lf.first + k]);
                ++n_leaves;
            }
            node_bytes = reinterpret_cast<uint8_t*>(&out.nodes[(size_t)it.addr * 4]);
            node_bytes[24 + c] = meta;
        }
        float* n = &out.nodes[(size_t)it.addr * 4];
        n[0] = lo[0];
        n[1] = lo[1];
        n[2] = lo[2];
        uint8_t* w = reinterpret_cast<uint8_t*>(&n[3]);
        w[0] = (uint8_t)e[0];
        w[1] = (uint8_t)e[1];
        w[2] = (uint8_t)e[2];
        w[3] = imask;
        n[4] = int_bits(child_base);
        n[5] = int_bits(tri_base);
        ++n_nodes;
    }
    out.node_count = n_nodes;
    out.leaf_count = n_leaves;
}

}  // namespace rq
