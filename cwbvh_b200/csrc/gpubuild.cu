// CWBVH built on the GPU from device-resident triangles, for scenes that must
// be ready quickly (a new scene admitted into a server) rather than traced
// at the best speed: a binary BVH over the Morton-ordered triangles (Karras's
// radix tree, or locally-ordered clustering), optional treelet passes, then
// a cost-optimal collapse into 8-wide nodes written directly in the CWBVH
// node format, with Woop rows and the primitive map, all on one stream.
//
//  1. centroid bounds (reduction), Morton code of each centroid above the
//     triangle number (unique 64-bit keys: ceil(log2 n) index bits, the rest,
//     up to 21 per axis, for the code), radix sort;
//  2. the binary tree: either internal node i of the radix tree over the
//     sorted keys, its key range and split from the longest common prefixes
//     (Karras, "Maximizing Parallelism in the Construction of BVHs, Octrees,
//     and k-d Trees", HPG 2012), with boxes and triangle counts bottom-up
//     (each leaf walks to the root and the second thread to reach a node
//     completes it, one atomic per node); or rounds of locally-ordered
//     clustering (see ploc_tree);
//  3. optional treelet restructuring passes (see restructure);
//  4. the host builder's cost-optimal collapse (dynamic programme over 1..8
//     slots per binary node, bottom-up), then level by level from the root
//     each 8-wide node's slots as it chose them; children with at most 3
//     triangles become leaves, the others 8-wide nodes of the next level.
//     Slots are assigned by the same octant rule as the host converter,
//     boxes quantized the same way, inner children get one contiguous block
//     and leaf triangles one contiguous run per node.
//
// The tree is a valid CWBVH for every trace kernel; it is not the host
// builder's (no spatial splits, different binary tree), so traversal is
// slower and the bytes differ.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "runtime.h"

namespace rq {
namespace {

struct BNode {
    int32_t left, right;  // >= 0: internal node, < 0: leaf ~(sorted position)
    int32_t parent;       // -1 at the root
    int32_t count;        // triangles below
    float lo[3], hi[3];
    float cost;           // SAH cost of the subtree
};

// SAH weights of the treelet restructuring (Karras and Aila 2013).
constexpr float kCt = 1.2f;  // per node
constexpr float kCi = 1.0f;  // per triangle

__device__ inline unsigned f2ord(float f) {
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ inline float ord2f(unsigned u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }

__device__ inline float3 vtx(const float* v, int32_t k) {
    const int64_t o = 3 * (int64_t)k;
    return make_float3(v[o], v[o + 1], v[o + 2]);
}

__device__ inline void tri_box(const float* v, const int32_t* idx, int64_t t, float lo[3], float hi[3]) {
    const float3 a = vtx(v, idx[3 * t]), b = vtx(v, idx[3 * t + 1]), c = vtx(v, idx[3 * t + 2]);
    lo[0] = fminf(a.x, fminf(b.x, c.x)); hi[0] = fmaxf(a.x, fmaxf(b.x, c.x));
    lo[1] = fminf(a.y, fminf(b.y, c.y)); hi[1] = fmaxf(a.y, fmaxf(b.y, c.y));
    lo[2] = fminf(a.z, fminf(b.z, c.z)); hi[2] = fmaxf(a.z, fmaxf(b.z, c.z));
}

// Sets *bad when an index is outside [0, nv): nothing else reads vertices
// through indices that have not passed this check.
__global__ void check_indices_kernel(const int32_t* idx, int64_t n3, int64_t nv, unsigned* bad) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n3; q += (int64_t)gridDim.x * blockDim.x)
        if (idx[q] < 0 || (int64_t)idx[q] >= nv) atomicOr(bad, 1u);
}

// ---- Triangle pre-splitting (the splitting stage of Karras and Aila, "Fast
// Parallel Construction of High-Quality Bounding Volume Hierarchies", HPG
// 2013, section 5).  A triangle whose box is much larger than the triangle
// itself (a sliver lying across the axes) is cut into several references
// along the planes of a 1024^3 grid over the scene, the most important plane
// first, so that the tree stages see tight boxes.  Each triangle receives
// pieces in proportion to its priority (2^m * wasted area)^(1/3), where m is
// the Morton level of the most important grid plane its box crosses and the
// wasted area is its box's half area minus the least half area boxes of its
// pieces can reach; the budget caps the extra pieces.  The references go to
// the tree stages as a "box mesh": a reference with box [lo, hi] is the
// triangle (lo, hi, hi), whose bounds are that box, so those stages read
// reference boxes through the same code as triangle boxes.  Only the Woop
// rows and the primitive map go back to the triangle.
constexpr int kSplitGridBits = 10;
constexpr int kMaxPieces = 32;

struct SplitGrid {
    float b0[3], ext[3];
};

__device__ inline SplitGrid split_grid(const unsigned* sb) {
    SplitGrid g;
    for (int a = 0; a < 3; ++a) {
        g.b0[a] = ord2f(sb[a]);
        g.ext[a] = ord2f(sb[3 + a]) - g.b0[a];
    }
    return g;
}

__device__ inline int grid_cell(const SplitGrid& g, int a, float x) {
    const float f = (x - g.b0[a]) / g.ext[a] * (float)(1 << kSplitGridBits);
    return (int)fminf(fmaxf(floorf(f), 0.f), (float)((1 << kSplitGridBits) - 1));
}

// The most important grid plane strictly inside [lo, hi]: the highest bit in
// which the cells of lo and hi differ, x before y before z at equal bits (the
// Morton order).  Returns its Morton level (3 * bit + 2 - axis) or -1.
__device__ int split_plane(const SplitGrid& g, const float lo[3], const float hi[3], int& axis, float& pos) {
    int best = -1;
    for (int a = 0; a < 3; ++a) {
        if (!(g.ext[a] > 0.f)) continue;
        const int q0 = grid_cell(g, a, lo[a]), q1 = grid_cell(g, a, hi[a]);
        if (q0 >= q1) continue;
        const int bit = 31 - __clz(q0 ^ q1);
        const int level = 3 * bit + 2 - a;
        if (level <= best) continue;
        const int cell = (q1 >> bit) << bit;  // first cell above the plane
        const float p = g.b0[a] + g.ext[a] * ((float)cell / (float)(1 << kSplitGridBits));
        if (!(p > lo[a] && p < hi[a])) continue;
        best = level;
        axis = a;
        pos = p;
    }
    return best;
}

// Scene bounds of the triangle boxes as order-preserving unsigned min / max.
__global__ void scene_bounds_kernel(const float* v, const int32_t* idx, int64_t n, unsigned* sb) {
    unsigned mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int32_t* ti = idx + 3 * t;
        for (int c = 0; c < 3; ++c) {
            const float3 p = vtx(v, ti[c]);
            const unsigned u[3] = {f2ord(p.x), f2ord(p.y), f2ord(p.z)};
            for (int a = 0; a < 3; ++a) {
                mn[a] = min(mn[a], u[a]);
                mx[a] = max(mx[a], u[a]);
            }
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xFFFFFFFFu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xFFFFFFFFu, mx[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(sb + a, mn[a]);
            atomicMax(sb + 3 + a, mx[a]);
        }
}

__device__ inline float half_area3(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    return dx * dy + dy * dz + dz * dx;
}

// Priority of each triangle.  The box of a piece of a flat patch with unit
// normal n and area A has half area at least 2 A (|nx| + |ny| + |nz|), which
// is |c.x| + |c.y| + |c.z| for the whole triangle, c = (b - a) x (c - a);
// the box's half area above that is what splitting can remove.
__global__ void split_priority_kernel(const float* v, const int32_t* idx, int64_t n, const unsigned* sb,
                                      float* prio) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t* ti = idx + 3 * t;
    const float3 a = vtx(v, ti[0]), b = vtx(v, ti[1]), c = vtx(v, ti[2]);
    const float lo[3] = {fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z))};
    const float hi[3] = {fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z))};
    const float ex = b.x - a.x, ey = b.y - a.y, ez = b.z - a.z;
    const float fx = c.x - a.x, fy = c.y - a.y, fz = c.z - a.z;
    const float ideal = fabsf(ey * fz - ez * fy) + fabsf(ez * fx - ex * fz) + fabsf(ex * fy - ey * fx);
    const float waste = half_area3(lo, hi) - ideal;
    const SplitGrid g = split_grid(sb);
    int axis = 0;
    float pos = 0.f;
    const int level = split_plane(g, lo, hi, axis, pos);
    prio[t] = (level < 0 || !(waste > 0.f)) ? 0.f : exp2f((float)level / 3.f) * cbrtf(waste);
}

// Pieces per triangle: 1 + its share of the `extra` budget, at most kMaxPieces.
__global__ void split_count_kernel(const float* prio, int64_t n, const float* sum, double extra, int64_t* pieces) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const double s = (double)*sum;
    const double share = s > 0.0 ? floor(extra * (double)prio[t] / s) : 0.0;
    pieces[t] = 1 + (int64_t)fmin(share, (double)(kMaxPieces - 1));
}

// The part of triangle (a, b, c) on one side of the plane x[axis] = p (upper
// side when `upper`), bounded in double and rounded outwards, clipped to box
// [blo, bhi].  Returns false when that part misses the box.
__device__ bool clip_side(const double3 (&tri)[3], int axis, double p, bool upper, const float blo[3],
                          const float bhi[3], float lo[3], float hi[3]) {
    double mn[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, mx[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    auto comp = [](const double3& q, int a) { return a == 0 ? q.x : (a == 1 ? q.y : q.z); };
    auto add = [&](double x, double y, double z) {
        mn[0] = fmin(mn[0], x); mx[0] = fmax(mx[0], x);
        mn[1] = fmin(mn[1], y); mx[1] = fmax(mx[1], y);
        mn[2] = fmin(mn[2], z); mx[2] = fmax(mx[2], z);
    };
    bool any = false;
    for (int i = 0; i < 3; ++i) {
        const double3& q = tri[i];
        const double qi = comp(q, axis);
        if (upper ? qi >= p : qi <= p) {
            add(q.x, q.y, q.z);
            any = true;
        }
        const double3& r = tri[(i + 1) % 3];
        const double ri = comp(r, axis);
        if ((qi < p && ri > p) || (qi > p && ri < p)) {
            const double s = (p - qi) / (ri - qi);
            double x = q.x + s * (r.x - q.x), y = q.y + s * (r.y - q.y), z = q.z + s * (r.z - q.z);
            if (axis == 0) x = p; else if (axis == 1) y = p; else z = p;
            add(x, y, z);
            any = true;
        }
    }
    if (!any) return false;
    for (int a = 0; a < 3; ++a) {
        lo[a] = fmaxf(__double2float_rd(mn[a]), blo[a]);
        hi[a] = fminf(__double2float_ru(mx[a]), bhi[a]);
        if (!(lo[a] <= hi[a])) return false;
    }
    return true;
}

// Cuts triangle t into pieces[t] references at off[t]: the box mesh (two
// corners per reference in rv, the triangle (2r, 2r + 1, 2r + 1) in ri) and
// the triangle of each reference (rtri).  Pieces are taken depth-first, the
// plane of each cut by split_plane, the pieces of a box shared between its
// two sides by their half areas; a box no plane cuts is one reference and
// any slots left over repeat the last reference.
struct SplitEntry {
    float lo[3], hi[3];
    int count;
};

__global__ void split_kernel(const float* v, const int32_t* idx, int64_t n, const unsigned* sb,
                             const int64_t* pieces, const int64_t* off, float* rv, int32_t* ri, int32_t* rtri) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int32_t* ti = idx + 3 * t;
    double3 tri[3];
    float lo[3], hi[3];
    for (int c = 0; c < 3; ++c) {
        const float3 p = vtx(v, ti[c]);
        tri[c] = make_double3(p.x, p.y, p.z);
    }
    for (int a = 0; a < 3; ++a) {
        const float x0 = a == 0 ? (float)tri[0].x : (a == 1 ? (float)tri[0].y : (float)tri[0].z);
        const float x1 = a == 0 ? (float)tri[1].x : (a == 1 ? (float)tri[1].y : (float)tri[1].z);
        const float x2 = a == 0 ? (float)tri[2].x : (a == 1 ? (float)tri[2].y : (float)tri[2].z);
        lo[a] = fminf(x0, fminf(x1, x2));
        hi[a] = fmaxf(x0, fmaxf(x1, x2));
    }
    const int total = (int)(pieces[t] < kMaxPieces ? pieces[t] : kMaxPieces);
    const int64_t base = off[t];
    const SplitGrid g = split_grid(sb);
    SplitEntry st[kMaxPieces];
    int sp = 0, emitted = 0, steps = 0;
    st[sp++] = SplitEntry{{lo[0], lo[1], lo[2]}, {hi[0], hi[1], hi[2]}, total};
    float last[6] = {lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]};
    auto emit = [&](const float* elo, const float* ehi) {
        if (emitted >= total) return;
        const int64_t r = base + emitted++;
        for (int a = 0; a < 3; ++a) {
            rv[6 * r + a] = elo[a];
            rv[6 * r + 3 + a] = ehi[a];
            last[a] = elo[a];
            last[3 + a] = ehi[a];
        }
        ri[3 * r] = (int32_t)(2 * r);
        ri[3 * r + 1] = (int32_t)(2 * r + 1);
        ri[3 * r + 2] = (int32_t)(2 * r + 1);
        rtri[r] = (int32_t)t;
    };
    while (sp > 0 && emitted < total) {
        const SplitEntry e = st[--sp];
        int axis = 0;
        float pos = 0.f;
        if (e.count == 1 || ++steps > 4 * kMaxPieces || split_plane(g, e.lo, e.hi, axis, pos) < 0) {
            emit(e.lo, e.hi);
            continue;
        }
        SplitEntry L, R;
        const bool okl = clip_side(tri, axis, (double)pos, false, e.lo, e.hi, L.lo, L.hi);
        const bool okr = clip_side(tri, axis, (double)pos, true, e.lo, e.hi, R.lo, R.hi);
        if (!okl && !okr) {
            emit(e.lo, e.hi);
            continue;
        }
        if (!okl || !okr) {  // all pieces to the one side that holds the triangle
            SplitEntry& o = okl ? L : R;
            o.count = e.count;
            st[sp++] = o;
            continue;
        }
        const float al = half_area3(L.lo, L.hi), ar = half_area3(R.lo, R.hi);
        int cl = (al + ar > 0.f) ? __float2int_rn((float)e.count * al / (al + ar)) : e.count / 2;
        cl = max(1, min(e.count - 1, cl));
        L.count = cl;
        R.count = e.count - cl;
        st[sp++] = R;  // counts on the stack never exceed total <= kMaxPieces entries
        st[sp++] = L;
    }
    while (emitted < total) emit(last, last + 3);
}

// Centroid bounds as order-preserving unsigned min / max (6 words).
__global__ void centroid_bounds_kernel(const float* v, const int32_t* idx, int64_t n, unsigned* ob) {
    unsigned mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        float lo[3], hi[3];
        tri_box(v, idx, t, lo, hi);
        for (int a = 0; a < 3; ++a) {
            const unsigned c = f2ord(0.5f * (lo[a] + hi[a]));
            mn[a] = min(mn[a], c);
            mx[a] = max(mx[a], c);
        }
    }
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xFFFFFFFFu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xFFFFFFFFu, mx[a], o));
        }
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) {
            atomicMin(ob + a, mn[a]);
            atomicMax(ob + 3 + a, mx[a]);
        }
}

// Spreads the low 21 bits of x to every third bit.
__device__ inline uint64_t spread3(uint64_t x) {
    x &= 0x1FFFFFull;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// key = Morton code of the centroid (`axis_bits` per axis) above the
// triangle number (`idx_bits`): unique, and as fine a grid as 64 bits allow.
__global__ void morton_kernel(const float* v, const int32_t* idx, int64_t n, const unsigned* ob, int axis_bits,
                              int idx_bits, uint64_t* keys) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float lo[3], hi[3];
    tri_box(v, idx, t, lo, hi);
    const float cells = (float)(1u << axis_bits);
    uint64_t q[3];
    for (int a = 0; a < 3; ++a) {
        const float b0 = ord2f(ob[a]), b1 = ord2f(ob[3 + a]);
        const float ext = b1 - b0;
        float f = ext > 0.f ? (0.5f * (lo[a] + hi[a]) - b0) / ext : 0.f;
        f = fminf(fmaxf(f, 0.f), 1.f);
        q[a] = min((uint64_t)((1u << axis_bits) - 1), (uint64_t)(f * cells));
    }
    const uint64_t m = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    keys[t] = (m << idx_bits) | (uint64_t)t;
}

__device__ inline int delta(const uint64_t* k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    return __clzll((long long)(k[i] ^ k[j]));
}

// Internal node i of the radix tree (Karras 2012, section 4).
__global__ void radix_tree_kernel(const uint64_t* k, int64_t n, BNode* nodes, int32_t* leaf_parent) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = delta(k, n, i, i + 1) - delta(k, n, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = delta(k, n, i, i - d);
    int64_t lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax *= 2;
    int64_t l = 0;
    for (int64_t t = lmax / 2; t >= 1; t /= 2)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    const int64_t j = i + l * d;
    const int dnode = delta(k, n, i, j);
    int64_t s = 0;
    for (int64_t div = 2;; div *= 2) {
        const int64_t t = (l + div - 1) / div;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    const int64_t gamma = i + s * d + min(d, 0);
    const int64_t lo = min(i, j), hi = max(i, j);
    BNode& nd = nodes[i];
    nd.left = lo == gamma ? ~(int32_t)gamma : (int32_t)gamma;
    nd.right = hi == gamma + 1 ? ~(int32_t)(gamma + 1) : (int32_t)(gamma + 1);
    if (nd.left >= 0) nodes[nd.left].parent = (int32_t)i;
    else leaf_parent[gamma] = (int32_t)i;
    if (nd.right >= 0) nodes[nd.right].parent = (int32_t)i;
    else leaf_parent[gamma + 1] = (int32_t)i;
    if (i == 0) nd.parent = -1;
}

// The triangle of a sorted key: its low idx_bits bits (idx_mask).
__device__ inline int64_t key_tri(const uint64_t* k, int64_t pos, uint64_t idx_mask) {
    return (int64_t)(k[pos] & idx_mask);
}

// Half the surface area of a box, and the SAH cost of a node over its two
// children, with every rounding explicit: the treelet kernels (one thread or
// one warp per treelet) compute the same costs bit for bit.
__device__ inline float half_area(const float lo[3], const float hi[3]) {
    const float dx = __fsub_rn(hi[0], lo[0]), dy = __fsub_rn(hi[1], lo[1]), dz = __fsub_rn(hi[2], lo[2]);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}
__device__ inline float node_cost(float area, float c0, float c1) {
    return __fadd_rn(__fadd_rn(__fmul_rn(kCt, area), c0), c1);
}

__device__ inline void child_box(const BNode* nodes, const uint64_t* k, uint64_t idx_mask, const float* v,
                                 const int32_t* idx, int32_t code, float lo[3], float hi[3], int32_t& count,
                                 float* cost = nullptr) {
    if (code >= 0) {
        const volatile BNode& c = nodes[code];
        for (int a = 0; a < 3; ++a) { lo[a] = c.lo[a]; hi[a] = c.hi[a]; }
        count = c.count;
        if (cost) *cost = c.cost;
    } else {
        tri_box(v, idx, key_tri(k, ~code, idx_mask), lo, hi);
        count = 1;
        if (cost) *cost = __fmul_rn(kCi, half_area(lo, hi));
    }
}

// Boxes and counts bottom-up: the second of a node's two children to arrive
// completes it and goes on to the parent.
__global__ void boxes_kernel(const uint64_t* k, uint64_t idx_mask, int64_t n, const float* v, const int32_t* idx,
                             BNode* nodes, const int32_t* leaf_parent, int32_t* arrivals) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int32_t node = leaf_parent[p];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;  // the sibling finishes this node
        __threadfence();
        float l0[3], h0[3], l1[3], h1[3], k0, k1;
        int32_t c0, c1;
        child_box(nodes, k, idx_mask, v, idx, nodes[node].left, l0, h0, c0, &k0);
        child_box(nodes, k, idx_mask, v, idx, nodes[node].right, l1, h1, c1, &k1);
        volatile BNode& nd = nodes[node];
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(l0[a], l1[a]);
            hi[a] = fmaxf(h0[a], h1[a]);
            nd.lo[a] = lo[a];
            nd.hi[a] = hi[a];
        }
        nd.count = c0 + c1;
        nd.cost = node_cost(half_area(lo, hi), k0, k1);
        node = nodes[node].parent;
    }
}

// ---- Treelet restructuring (Karras and Aila, "Fast Parallel Construction of
// High-Quality Bounding Volume Hierarchies", HPG 2013): bottom-up again, each
// node with at least `min_count` triangles forms a treelet by expanding its
// largest-area leaf until it has 7 leaves, finds the SAH-optimal binary tree
// over those leaves by dynamic programming over the 127 leaf subsets, and
// rebuilds the treelet with it (reusing its 6 internal nodes) when cheaper.
// Treelets of different nodes being restructured at once are disjoint: a node
// is processed only when both its children are final.
constexpr int kTreeletLeaves = 7;

// Node fields other threads of the same launch may have rewritten are read
// from L2 (ld.cg), never from a possibly stale L1 line.
__device__ inline int32_t ld_left(const BNode* nodes, int32_t x) { return __ldcg(&nodes[x].left); }
__device__ inline int32_t ld_right(const BNode* nodes, int32_t x) { return __ldcg(&nodes[x].right); }
__device__ inline int32_t ld_parent(const BNode* nodes, int32_t x) { return __ldcg(&nodes[x].parent); }

__device__ void restructure(BNode* nodes, const uint64_t* k, uint64_t idx_mask, const float* v, const int32_t* idx,
                            int32_t* leaf_parent, int32_t root) {
    int32_t inner[kTreeletLeaves - 1], leaf[kTreeletLeaves];
    float larea[kTreeletLeaves];
    int n_in = 1, n_leaf = 2;
    inner[0] = root;
    leaf[0] = ld_left(nodes, root);
    leaf[1] = ld_right(nodes, root);
    float llo[kTreeletLeaves][3], lhi[kTreeletLeaves][3], lcost[kTreeletLeaves];
    int32_t lcnt[kTreeletLeaves];
    for (int q = 0; q < 2; ++q) {
        child_box(nodes, k, idx_mask, v, idx, leaf[q], llo[q], lhi[q], lcnt[q], &lcost[q]);
        larea[q] = half_area(llo[q], lhi[q]);
    }
    while (n_leaf < kTreeletLeaves) {
        int best = -1;
        float ba = -1.f;
        for (int q = 0; q < n_leaf; ++q)
            if (leaf[q] >= 0 && larea[q] > ba) { ba = larea[q]; best = q; }
        if (best < 0) break;
        const int32_t x = leaf[best];
        inner[n_in++] = x;
        const int32_t l = ld_left(nodes, x), r = ld_right(nodes, x);
        leaf[best] = l;
        child_box(nodes, k, idx_mask, v, idx, l, llo[best], lhi[best], lcnt[best], &lcost[best]);
        larea[best] = half_area(llo[best], lhi[best]);
        leaf[n_leaf] = r;
        child_box(nodes, k, idx_mask, v, idx, r, llo[n_leaf], lhi[n_leaf], lcnt[n_leaf], &lcost[n_leaf]);
        larea[n_leaf] = half_area(llo[n_leaf], lhi[n_leaf]);
        ++n_leaf;
    }
    if (n_leaf < 3) return;
    const int full = (1 << n_leaf) - 1;
    // Subset boxes are recomputed from the leaves when needed instead of
    // kept per subset: min / max are exact in any order, so the boxes are
    // the same, and the per-thread table shrinks from 3.7 KB to 640 B.
    auto subset_box = [&](int S, float lo[3], float hi[3]) {
        for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
        for (int q = 0; q < n_leaf; ++q)
            if (S & (1 << q))
                for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], llo[q][a]); hi[a] = fmaxf(hi[a], lhi[q][a]); }
    };
    float cost[1 << kTreeletLeaves];
    uint8_t part[1 << kTreeletLeaves];
    for (int S = 1; S <= full; ++S) {
        const int low = __ffs(S) - 1;
        const int rest = S & (S - 1);
        if (rest == 0) {
            cost[S] = lcost[low];
            part[S] = 0;
            continue;
        }
        float slo[3], shi[3];
        subset_box(S, slo, shi);
        float best = FLT_MAX;
        int bp = 0;
        // partitions {P, S \ P} with the lowest leaf in P, P != S
        for (int P = (S - 1) & S; P > 0; P = (P - 1) & S) {
            if (!(P & (1 << low))) continue;
            const float c = __fadd_rn(cost[P], cost[S ^ P]);
            if (c < best) { best = c; bp = P; }
        }
        cost[S] = __fadd_rn(__fmul_rn(kCt, half_area(slo, shi)), best);
        part[S] = (uint8_t)bp;
    }
    if (!(cost[full] < 0.999f * __ldcg(&nodes[root].cost))) return;
    // every subset the new tree splits must have a split (finite costs); check
    // before writing anything
    {
        int st[kTreeletLeaves], sp = 0;
        st[sp++] = full;
        while (sp > 0) {
            const int S = st[--sp];
            const int P = part[S];
            if (P == 0 || (P & ~S) != 0 || P == S) return;
            if (P & (P - 1)) st[sp++] = P;
            if ((S ^ P) & ((S ^ P) - 1)) st[sp++] = S ^ P;
            if (sp > kTreeletLeaves - 1) return;
        }
    }
    // rebuild top-down: subset -> node, internal nodes taken from `inner`
    int32_t st_set[kTreeletLeaves], st_node[kTreeletLeaves];
    int sp = 0, used = 1;
    st_set[sp] = full;
    st_node[sp++] = root;
    while (sp > 0) {
        --sp;
        const int S = st_set[sp];
        const int32_t nd = st_node[sp];
        const int P = part[S];
        const int side[2] = {P, S ^ P};
        int32_t code[2];
        for (int c = 0; c < 2; ++c) {
            const int T = side[c];
            if ((T & (T - 1)) == 0) {  // one leaf of the treelet
                code[c] = leaf[__ffs(T) - 1];
                if (code[c] >= 0) nodes[code[c]].parent = nd;
                else leaf_parent[~code[c]] = nd;
            } else {
                const int32_t ni = inner[used++];
                code[c] = ni;
                nodes[ni].parent = nd;
                st_set[sp] = T;
                st_node[sp++] = ni;
            }
        }
        BNode& b = nodes[nd];
        b.left = code[0];
        b.right = code[1];
        float slo[3], shi[3];
        subset_box(S, slo, shi);
        for (int a = 0; a < 3; ++a) { b.lo[a] = slo[a]; b.hi[a] = shi[a]; }
        int32_t cnt = 0;
        for (int q = 0; q < n_leaf; ++q)
            if (S & (1 << q)) cnt += lcnt[q];
        b.count = cnt;
        b.cost = cost[S];
    }
}

__global__ void treelet_kernel(const uint64_t* k, uint64_t idx_mask, int64_t n, const float* v, const int32_t* idx,
                               BNode* nodes, int32_t* leaf_parent, int32_t* arrivals, int min_count) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int32_t node = leaf_parent[p];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;
        __threadfence();
        // this node's cost from its (final) children, then its treelet
        float l0[3], h0[3], l1[3], h1[3], k0, k1;
        int32_t c0, c1;
        child_box(nodes, k, idx_mask, v, idx, ld_left(nodes, node), l0, h0, c0, &k0);
        child_box(nodes, k, idx_mask, v, idx, ld_right(nodes, node), l1, h1, c1, &k1);
        volatile BNode& nd = nodes[node];
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) { lo[a] = fminf(l0[a], l1[a]); hi[a] = fmaxf(h0[a], h1[a]); }
        nd.cost = node_cost(half_area(lo, hi), k0, k1);
        if (c0 + c1 >= min_count) restructure(nodes, k, idx_mask, v, idx, leaf_parent, node);
        node = ld_parent(nodes, node);
    }
}

// ---- The same restructuring with a warp per treelet (the parallel form of
// Karras and Aila, section 4.2).  Lanes walk up the tree as in
// treelet_kernel; at each step the nodes whose treelets are due are taken one
// at a time by the whole warp: lane q holds leaf q while the treelet grows,
// the subsets of one size are costed by different lanes (smaller subsets
// first, so every partition's two parts are ready; a subset's box is its
// box without its highest leaf, kept in shared memory, joined with that
// leaf's), and the 63 partitions of the 7-leaf set are spread over the lanes
// and reduced with shuffles.  Every subset's cost is the same expression in
// the same order as in restructure(), and the chosen partition is the first
// minimum in its enumeration order there, so the trees are identical.
constexpr unsigned kWarpAll = 0xFFFFFFFFu;

struct SubsetTable {
    uint8_t set[127];   // the subsets of 7 leaves by size, then value
    uint8_t start[9];   // first entry of each size (start[8] = 127)
};
constexpr SubsetTable make_subset_table() {
    SubsetTable t{};
    int k = 0;
    for (int size = 1; size <= 7; ++size) {
        t.start[size] = (uint8_t)k;
        for (int S = 1; S < 128; ++S) {
            int c = 0;
            for (int b = 0; b < 7; ++b) c += (S >> b) & 1;
            if (c == size) t.set[k++] = (uint8_t)S;
        }
    }
    t.start[0] = 0;
    t.start[8] = (uint8_t)k;
    return t;
}
__constant__ SubsetTable c_subsets = make_subset_table();

struct TreeletSmem {
    float llo[kTreeletLeaves][3], lhi[kTreeletLeaves][3], lcost[kTreeletLeaves];
    int32_t lcnt[kTreeletLeaves], leaf[kTreeletLeaves], inner[kTreeletLeaves - 1];
    float cost[1 << kTreeletLeaves];
    float slo[1 << kTreeletLeaves][3], shi[1 << kTreeletLeaves][3];  // subset boxes
    uint8_t part[1 << kTreeletLeaves];
};

// The i-th partition {P, S ^ P} of S in restructure()'s order: P holds the
// lowest leaf of S, and P runs down from S - 1 over the subsets of S.
__device__ inline int nth_partition(int S, int i) {
    const int low = S & -S;
    const int R = S ^ low;  // the other leaves
    // Q = the i-th largest proper subset of R: the bits of (2^|R| - 2 - i)
    // deposited into the positions of R.
    const int nb = __popc(R);
    int v = (1 << nb) - 2 - i, Q = 0, r = R;
    for (int b = 0; b < nb; ++b) {
        const int bit = r & -r;
        if (v & (1 << b)) Q |= bit;
        r ^= bit;
    }
    return low | Q;
}

// The box of subset S (two or more leaves) from the box of S without its
// highest leaf, already in the table, and that leaf's box; min / max are
// exact in any order, so it equals restructure()'s box of the same leaves.
__device__ void subset_box_s(TreeletSmem& t, int S, float lo[3], float hi[3]) {
    const int high = 31 - __clz(S);
    const int R = S & ~(1 << high);
    for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(t.slo[R][a], t.llo[high][a]);
        hi[a] = fmaxf(t.shi[R][a], t.lhi[high][a]);
        t.slo[S][a] = lo[a];
        t.shi[S][a] = hi[a];
    }
}

// The whole warp restructures the treelet rooted at `root` (warp-uniform).
__device__ void restructure_warp(BNode* nodes, const uint64_t* k, uint64_t idx_mask, const float* v,
                                 const int32_t* idx, int32_t* leaf_parent, int32_t root, float root_cost,
                                 TreeletSmem& t) {
    const unsigned lane = threadIdx.x & 31u;
    // Grow the treelet: lane q holds leaf q.
    int32_t my_leaf = -1;
    float mlo[3] = {0.f, 0.f, 0.f}, mhi[3] = {0.f, 0.f, 0.f}, mcost = 0.f, marea = -1.f;
    int32_t mcnt = 0;
    int n_in = 1, n_leaf = 2;
    if (lane < 2) {
        my_leaf = lane == 0 ? ld_left(nodes, root) : ld_right(nodes, root);
        child_box(nodes, k, idx_mask, v, idx, my_leaf, mlo, mhi, mcnt, &mcost);
        marea = half_area(mlo, mhi);
    }
    if (lane == 0) t.inner[0] = root;
    while (n_leaf < kTreeletLeaves) {
        // the first leaf of the largest area that is a node (restructure()'s scan)
        float a = ((int)lane < n_leaf && my_leaf >= 0) ? marea : -1.f;
        int best = ((int)lane < n_leaf && my_leaf >= 0) ? (int)lane : 64;
        for (int o = 16; o > 0; o >>= 1) {
            const float a2 = __shfl_xor_sync(kWarpAll, a, o);
            const int b2 = __shfl_xor_sync(kWarpAll, best, o);
            if (a2 > a || (a2 == a && b2 < best)) { a = a2; best = b2; }
        }
        if (best >= 64 || !(a > -1.f)) break;
        const int32_t x = __shfl_sync(kWarpAll, my_leaf, best);
        if (lane == 0) t.inner[n_in] = x;
        ++n_in;
        if ((int)lane == best || (int)lane == n_leaf) {
            my_leaf = (int)lane == best ? ld_left(nodes, x) : ld_right(nodes, x);
            child_box(nodes, k, idx_mask, v, idx, my_leaf, mlo, mhi, mcnt, &mcost);
            marea = half_area(mlo, mhi);
        }
        ++n_leaf;
    }
    if (n_leaf < 3) return;
    if ((int)lane < n_leaf) {
        for (int a = 0; a < 3; ++a) {
            t.llo[lane][a] = mlo[a];
            t.lhi[lane][a] = mhi[a];
            t.slo[1 << lane][a] = mlo[a];
            t.shi[1 << lane][a] = mhi[a];
        }
        t.lcost[lane] = mcost;
        t.lcnt[lane] = mcnt;
        t.leaf[lane] = my_leaf;
        t.cost[1 << lane] = mcost;
        t.part[1 << lane] = 0;
    }
    __syncwarp();
    const int full = (1 << n_leaf) - 1;
    for (int size = 2; size <= n_leaf; ++size) {
        const int first = c_subsets.start[size], end = c_subsets.start[size + 1];
        if (size < 7) {
            // one subset per lane
            for (int e = first + (int)lane; e < end; e += 32) {
                const int S = c_subsets.set[e];
                if (S > full) continue;
                float slo[3], shi[3];
                subset_box_s(t, S, slo, shi);
                const int low = __ffs(S) - 1;
                float bc = FLT_MAX;
                int bp = 0;
                for (int P = (S - 1) & S; P > 0; P = (P - 1) & S) {
                    if (!(P & (1 << low))) continue;
                    const float c = __fadd_rn(t.cost[P], t.cost[S ^ P]);
                    if (c < bc) { bc = c; bp = P; }
                }
                t.cost[S] = __fadd_rn(__fmul_rn(kCt, half_area(slo, shi)), bc);
                t.part[S] = (uint8_t)bp;
            }
        } else {
            // one subset at a time, its partitions over the lanes
            for (int e = first; e < end; ++e) {
                const int S = c_subsets.set[e];
                if (S > full) continue;
                const int n_part = (1 << (__popc(S) - 1)) - 1;
                float bc = FLT_MAX;
                int bi = 1 << 30;
                for (int i = (int)lane; i < n_part; i += 32) {
                    const int P = nth_partition(S, i);
                    const float c = __fadd_rn(t.cost[P], t.cost[S ^ P]);
                    if (c < bc) { bc = c; bi = i; }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const float c2 = __shfl_xor_sync(kWarpAll, bc, o);
                    const int i2 = __shfl_xor_sync(kWarpAll, bi, o);
                    if (c2 < bc || (c2 == bc && i2 < bi)) { bc = c2; bi = i2; }
                }
                if (lane == 0) {
                    float slo[3], shi[3];
                    subset_box_s(t, S, slo, shi);
                    t.cost[S] = __fadd_rn(__fmul_rn(kCt, half_area(slo, shi)), bc);
                    t.part[S] = (uint8_t)(bi < n_part ? nth_partition(S, bi) : 0);
                }
                __syncwarp();
            }
        }
        __syncwarp();
    }
    if (lane == 0 && t.cost[full] < 0.999f * root_cost) {
        // every subset the new tree splits must have a split (finite costs);
        // check before writing anything
        bool ok = true;
        {
            int st[kTreeletLeaves], sp = 0;
            st[sp++] = full;
            while (sp > 0 && ok) {
                const int S = st[--sp];
                const int P = t.part[S];
                if (P == 0 || (P & ~S) != 0 || P == S) { ok = false; break; }
                if (P & (P - 1)) st[sp++] = P;
                if ((S ^ P) & ((S ^ P) - 1)) st[sp++] = S ^ P;
                if (sp > kTreeletLeaves - 1) ok = false;
            }
        }
        if (ok) {
            // rebuild top-down: subset -> node, internal nodes taken from `inner`
            int32_t st_set[kTreeletLeaves], st_node[kTreeletLeaves];
            int sp = 0, used = 1;
            st_set[sp] = full;
            st_node[sp++] = root;
            while (sp > 0) {
                --sp;
                const int S = st_set[sp];
                const int32_t nd = st_node[sp];
                const int P = t.part[S];
                const int side[2] = {P, S ^ P};
                int32_t code[2];
                for (int c = 0; c < 2; ++c) {
                    const int T = side[c];
                    if ((T & (T - 1)) == 0) {
                        code[c] = t.leaf[__ffs(T) - 1];
                        if (code[c] >= 0) nodes[code[c]].parent = nd;
                        else leaf_parent[~code[c]] = nd;
                    } else {
                        const int32_t ni = t.inner[used++];
                        code[c] = ni;
                        nodes[ni].parent = nd;
                        st_set[sp] = T;
                        st_node[sp++] = ni;
                    }
                }
                BNode& b = nodes[nd];
                b.left = code[0];
                b.right = code[1];
                for (int a = 0; a < 3; ++a) { b.lo[a] = t.slo[S][a]; b.hi[a] = t.shi[S][a]; }
                int32_t cnt = 0;
                for (int q = 0; q < n_leaf; ++q)
                    if (S & (1 << q)) cnt += t.lcnt[q];
                b.count = cnt;
                b.cost = t.cost[S];
            }
            __threadfence();
        }
    }
    __syncwarp();
}

constexpr int kTreeletWarpBlock = 128;

__global__ void __launch_bounds__(kTreeletWarpBlock) treelet_warp_kernel(
        const uint64_t* k, uint64_t idx_mask, int64_t n, const float* v, const int32_t* idx, BNode* nodes,
        int32_t* leaf_parent, int32_t* arrivals, int min_count) {
    __shared__ TreeletSmem smem[kTreeletWarpBlock / 32];
    TreeletSmem& t = smem[threadIdx.x / 32];
    const unsigned lane = threadIdx.x & 31u;
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int32_t node = p < n ? leaf_parent[p] : -1;
    for (;;) {
        bool go = node >= 0;
        if (go) {
            __threadfence();
            if (atomicAdd(&arrivals[node], 1) == 0) go = false;  // the sibling's thread finishes this node
            __threadfence();
        }
        if (!go) node = -1;
        float cost = 0.f;
        bool due = false;
        if (go) {
            float l0[3], h0[3], l1[3], h1[3], k0, k1;
            int32_t c0, c1;
            child_box(nodes, k, idx_mask, v, idx, ld_left(nodes, node), l0, h0, c0, &k0);
            child_box(nodes, k, idx_mask, v, idx, ld_right(nodes, node), l1, h1, c1, &k1);
            volatile BNode& nd = nodes[node];
            float lo[3], hi[3];
            for (int a = 0; a < 3; ++a) { lo[a] = fminf(l0[a], l1[a]); hi[a] = fmaxf(h0[a], h1[a]); }
            cost = node_cost(half_area(lo, hi), k0, k1);
            nd.cost = cost;
            due = c0 + c1 >= min_count;
        }
        unsigned want = __ballot_sync(kWarpAll, due);
        while (want) {
            const int src = __ffs(want) - 1;
            want &= want - 1;
            const int32_t root = __shfl_sync(kWarpAll, node, src);
            const float rc = __shfl_sync(kWarpAll, cost, src);
            restructure_warp(nodes, k, idx_mask, v, idx, leaf_parent, root, rc, t);
        }
        if (go) node = ld_parent(nodes, node);
        if (__ballot_sync(kWarpAll, node >= 0) == 0u) break;
    }
}

// ---- Woop rows (the host woopify, with every rounding explicit so that the
// device gives the host's values for the same triangle).
__device__ void woopify_dev(float3 v0, float3 v1, float3 v2, float4* out) {
    const float3 e0 = make_float3(__fsub_rn(v0.x, v2.x), __fsub_rn(v0.y, v2.y), __fsub_rn(v0.z, v2.z));
    const float3 e1 = make_float3(__fsub_rn(v1.x, v2.x), __fsub_rn(v1.y, v2.y), __fsub_rn(v1.z, v2.z));
    const float3 nn = make_float3(__fsub_rn(__fmul_rn(e0.y, e1.z), __fmul_rn(e0.z, e1.y)),
                                  __fsub_rn(__fmul_rn(e0.z, e1.x), __fmul_rn(e0.x, e1.z)),
                                  __fsub_rn(__fmul_rn(e0.x, e1.y), __fmul_rn(e0.y, e1.x)));
    const double a[3][3] = {{e0.x, e1.x, nn.x}, {e0.y, e1.y, nn.y}, {e0.z, e1.z, nn.z}};
    const double t[3] = {v2.x, v2.y, v2.z};
    auto m2 = [](double p, double q, double r, double s) { return __dsub_rn(__dmul_rn(p, q), __dmul_rn(r, s)); };
    double c[3][3];
    c[0][0] = m2(a[1][1], a[2][2], a[1][2], a[2][1]);
    c[0][1] = m2(a[0][2], a[2][1], a[0][1], a[2][2]);
    c[0][2] = m2(a[0][1], a[1][2], a[0][2], a[1][1]);
    c[1][0] = m2(a[1][2], a[2][0], a[1][0], a[2][2]);
    c[1][1] = m2(a[0][0], a[2][2], a[0][2], a[2][0]);
    c[1][2] = m2(a[0][2], a[1][0], a[0][0], a[1][2]);
    c[2][0] = m2(a[1][0], a[2][1], a[1][1], a[2][0]);
    c[2][1] = m2(a[0][1], a[2][0], a[0][0], a[2][1]);
    c[2][2] = m2(a[0][0], a[1][1], a[0][1], a[1][0]);
    const double det = __dadd_rn(__dadd_rn(__dmul_rn(a[0][0], c[0][0]), __dmul_rn(a[0][1], c[1][0])),
                                 __dmul_rn(a[0][2], c[2][0]));
    if (det == 0.0 || !isfinite(det)) {
        out[0] = out[1] = out[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const double rdet = __ddiv_rn(1.0, det);
    double inv[3][4];
    for (int r = 0; r < 3; ++r) {
        for (int q = 0; q < 3; ++q) inv[r][q] = __dmul_rn(c[r][q], rdet);
        inv[r][3] = -__dadd_rn(__dadd_rn(__dmul_rn(inv[r][0], t[0]), __dmul_rn(inv[r][1], t[1])),
                               __dmul_rn(inv[r][2], t[2]));
    }
    float x0 = (float)inv[2][0];
    if (x0 == 0.0f) x0 = 0.0f;  // -0.0f would read as a BVH2 leaf terminator
    out[0] = make_float4(x0, (float)inv[2][1], (float)inv[2][2], (float)(-inv[2][3]));
    out[1] = make_float4((float)inv[0][0], (float)inv[0][1], (float)inv[0][2], (float)inv[0][3]);
    out[2] = make_float4((float)inv[1][0], (float)inv[1][1], (float)inv[1][2], (float)inv[1][3]);
}

struct Item {
    int32_t code;  // binary node (>= 0) or a single-triangle root (< 0)
    int32_t addr;  // 8-wide node index
};

struct Ctr {
    unsigned long long nodes;  // 8-wide nodes allocated
    unsigned long long tris;   // triangle slots allocated
    unsigned long long next;   // items of the next level
    unsigned int error;
};

// ---- Cost-optimal collapse into 8-wide nodes (the host builder's dynamic
// programme): for every binary node and k = 1..8 slots, the least
// surface-area cost of representing its subtree with at most k children of
// an 8-wide node -- one leaf (at most 3 triangles), an 8-wide node of its
// own, or the node opened with j slots to its left child and k - j to its
// right.  Computed bottom-up (the second child to finish completes a node);
// the expansion then replays the choices instead of opening the largest
// child greedily.
constexpr float kCollapseNode = 1.0f;  // per 8-wide node, times its area
constexpr float kCollapseLeaf = 0.3f;  // per triangle in a leaf, times the leaf's area

struct CollapseDP {
    float best[8];    // k = 1..8
    uint8_t how[8];   // 0 leaf, 1 own node, 2 + j opened with j slots to the left child
    uint8_t split8;   // slots to the left child when the node is an 8-wide node of its own
    uint8_t pad[7];
};

__global__ void collapse_dp_kernel(const uint64_t* k, uint64_t idx_mask, int64_t n, const float* v,
                                   const int32_t* idx, const BNode* nodes, const int32_t* leaf_parent,
                                   int32_t* arrivals, CollapseDP* dp) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int32_t node = leaf_parent[p];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1) == 0) return;  // the sibling finishes this node
        __threadfence();
        const int32_t c[2] = {__ldcg(&nodes[node].left), __ldcg(&nodes[node].right)};
        float cost[2][9], area[2];
        int32_t cnt[2];
        for (int q = 0; q < 2; ++q) {
            float lo[3], hi[3];
            child_box(nodes, k, idx_mask, v, idx, c[q], lo, hi, cnt[q]);
            area[q] = half_area(lo, hi);
            for (int kk = 1; kk <= 8; ++kk)
                cost[q][kk] = c[q] >= 0 ? __ldcg(&dp[c[q]].best[kk - 1]) : kCollapseLeaf * area[q];
        }
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = __ldcg(&nodes[node].lo[a]);
            hi[a] = __ldcg(&nodes[node].hi[a]);
        }
        const float av = half_area(lo, hi);
        const int32_t prims = cnt[0] + cnt[1];
        float open[9];
        uint8_t split[9];
        for (int kk = 2; kk <= 8; ++kk) {
            open[kk] = FLT_MAX;
            split[kk] = 1;
            for (int j = 1; j < kk; ++j) {
                const float cc = cost[0][j] + cost[1][kk - j];
                if (cc < open[kk]) { open[kk] = cc; split[kk] = (uint8_t)j; }
            }
        }
        CollapseDP d;
        const float as_node = kCollapseNode * av + open[8];
        const float as_leaf = prims <= 3 ? kCollapseLeaf * av * (float)prims : FLT_MAX;
        d.best[0] = fminf(as_leaf, as_node);
        d.how[0] = as_leaf <= as_node ? 0 : 1;
        for (int kk = 2; kk <= 8; ++kk) {
            d.best[kk - 1] = d.best[kk - 2];
            d.how[kk - 1] = d.how[kk - 2];
            if (open[kk] < d.best[kk - 1]) { d.best[kk - 1] = open[kk]; d.how[kk - 1] = (uint8_t)(2 + split[kk]); }
        }
        d.split8 = split[8];
        dp[node] = d;
        node = __ldcg(&nodes[node].parent);
    }
}

// Expands the binary nodes of one level into 8-wide nodes, their slots as
// the collapse chose them.
__global__ void expand_kernel(const Item* items, int64_t n_items, Item* next, int64_t next_cap, const BNode* nodes,
                              const uint64_t* k, uint64_t idx_mask, const float* v, const int32_t* idx,
                              const float* tv, const int32_t* tidx, const int32_t* ref_tri, float4* out_nodes,
                              int64_t node_cap, float4* woop, int32_t* prim, int64_t tri_cap, Ctr* ctr,
                              const CollapseDP* dp) {
    const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_items) return;
    const Item it = items[w];
    int32_t code[8];
    float clo[8][3], chi[8][3];
    int32_t cnt[8];
    int m = 0;
    if (it.code < 0) {  // one triangle: the root holds one leaf
        code[0] = it.code;
        child_box(nodes, k, idx_mask, v, idx, it.code, clo[0], chi[0], cnt[0]);
        m = 1;
    } else if (dp) {
        // the slots the collapse chose: (binary child, slots it fills), left first
        int32_t stc[16];
        int stk[16];
        int sp = 0;
        const BNode& b = nodes[it.code];
        const int s8 = dp[it.code].split8;
        stc[sp] = b.right; stk[sp++] = 8 - s8;
        stc[sp] = b.left; stk[sp++] = s8;
        while (sp > 0) {
            --sp;
            const int32_t x = stc[sp];
            const int kk = stk[sp];
            const int h = (x >= 0 && kk >= 1 && kk <= 8) ? dp[x].how[kk - 1] : 0;
            if (h >= 2) {
                const int j = h - 2;
                if (sp + 2 > 16 || j < 1 || j >= kk) {  // a table the recursion cannot follow
                    atomicOr(&ctr->error, 4u);
                    return;
                }
                stc[sp] = nodes[x].right; stk[sp++] = kk - j;
                stc[sp] = nodes[x].left; stk[sp++] = j;
            } else {
                if (m >= 8) {
                    atomicOr(&ctr->error, 4u);
                    return;
                }
                code[m] = x;
                child_box(nodes, k, idx_mask, v, idx, x, clo[m], chi[m], cnt[m]);
                ++m;
            }
        }
    } else {
        atomicOr(&ctr->error, 4u);  // an inner node needs the collapse table
        return;
    }
    // node box
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int c = 0; c < m; ++c)
        for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], clo[c][a]); hi[a] = fmaxf(hi[a], chi[c][a]); }
    // octant slots: cheapest (slot, child) pairs first, as the host converter
    float nc[3];
    for (int a = 0; a < 3; ++a) nc[a] = (lo[a] + hi[a]) * 0.5f;
    int slot_of[8], child_in[8];
    bool slot_free[8];
    for (int s = 0; s < 8; ++s) { slot_of[s] = -1; slot_free[s] = true; child_in[s] = -1; }
    for (;;) {
        float best = FLT_MAX;
        int bs = -1, bc = -1;
        for (int s = 0; s < 8; ++s) {
            if (!slot_free[s]) continue;
            const float dx = (s & 4) ? -1.f : 1.f, dy = (s & 2) ? -1.f : 1.f, dz = (s & 1) ? -1.f : 1.f;
            for (int c = 0; c < m; ++c) {
                if (slot_of[c] >= 0) continue;
                const float cx = __fsub_rn(__fmul_rn(__fadd_rn(clo[c][0], chi[c][0]), 0.5f), nc[0]);
                const float cy = __fsub_rn(__fmul_rn(__fadd_rn(clo[c][1], chi[c][1]), 0.5f), nc[1]);
                const float cz = __fsub_rn(__fmul_rn(__fadd_rn(clo[c][2], chi[c][2]), 0.5f), nc[2]);
                const float cost = __fadd_rn(__fadd_rn(__fmul_rn(cx, dx), __fmul_rn(cy, dy)), __fmul_rn(cz, dz));
                if (cost < best) { best = cost; bs = s; bc = c; }
            }
        }
        if (bs < 0) break;
        slot_free[bs] = false;
        slot_of[bc] = bs;
        child_in[bs] = bc;
    }
    // per-axis exponent, grown while a child's upper bound does not fit a byte
    int e[3];
    for (int a = 0; a < 3; ++a) {
        const float r = ceilf(log2f((hi[a] - lo[a]) / 255.0f));
        e[a] = isfinite(r) ? (int)fmaxf(-127.f, fminf(127.f, r)) : 0;
        for (;;) {
            const float scale = ldexpf(1.0f, e[a]);
            bool fits = true;
            for (int c = 0; c < m; ++c)
                if ((int)ceilf((chi[c][a] - lo[a]) / scale) > 255) fits = false;
            if (fits || e[a] >= 127) break;
            ++e[a];
        }
    }
    // allocations: inner children as one block, leaf triangles as one run
    int n_inner = 0, n_tris = 0;
    for (int c = 0; c < m; ++c) {
        if (cnt[c] > 3) ++n_inner;
        else n_tris += cnt[c];
    }
    const unsigned long long base = n_inner ? atomicAdd(&ctr->nodes, (unsigned long long)n_inner) : 0ull;
    const unsigned long long tbase = n_tris ? atomicAdd(&ctr->tris, (unsigned long long)n_tris) : 0ull;
    const unsigned long long qbase = n_inner ? atomicAdd(&ctr->next, (unsigned long long)n_inner) : 0ull;
    if (base + n_inner > (unsigned long long)node_cap || tbase + n_tris > (unsigned long long)tri_cap ||
        qbase + n_inner > (unsigned long long)next_cap) {
        atomicOr(&ctr->error, 1u);
        return;
    }
    float4 node[5];
    for (int q = 0; q < 5; ++q) node[q] = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned char* bytes = reinterpret_cast<unsigned char*>(node);
    uint8_t imask = 0;
    int inner = 0, leaf_tris = 0;
    for (int s = 0; s < 8; ++s) {
        const int c = child_in[s];
        if (c < 0) continue;
        for (int a = 0; a < 3; ++a) {
            const float scale = ldexpf(1.0f, e[a]);
            bytes[32 + s + 8 * a] = (uint8_t)(int)floorf((clo[c][a] - lo[a]) / scale);
            bytes[32 + s + 8 * (3 + a)] = (uint8_t)(int)ceilf((chi[c][a] - lo[a]) / scale);
        }
        if (cnt[c] > 3) {
            imask |= (uint8_t)(1u << s);
            bytes[24 + s] = (uint8_t)((1u << 5) | (24u + s));
            next[qbase + inner] = Item{code[c], (int32_t)(base + inner)};
            ++inner;
        } else {
            const uint32_t unary = cnt[c] == 1 ? 1u : (cnt[c] == 2 ? 3u : 7u);
            bytes[24 + s] = (uint8_t)((unary << 5) | ((uint32_t)leaf_tris & 31u));
            // the child's triangles: a leaf, or a subtree of at most 3
            int32_t st[4];
            int sp = 0;
            st[sp++] = code[c];
            while (sp > 0) {
                const int32_t x = st[--sp];
                if (leaf_tris >= n_tris || (x >= 0 && sp + 2 > 4)) {  // counts disagree with the tree
                    atomicOr(&ctr->error, 2u);
                    return;
                }
                if (x < 0) {
                    const int64_t ref = key_tri(k, ~x, idx_mask);
                    const int64_t tri = ref_tri ? (int64_t)ref_tri[ref] : ref;
                    const int64_t slot = (int64_t)tbase + leaf_tris;
                    const int32_t* ti = tidx + 3 * tri;
                    woopify_dev(vtx(tv, ti[0]), vtx(tv, ti[1]), vtx(tv, ti[2]), woop + 3 * slot);
                    prim[3 * slot] = (int32_t)tri;
                    prim[3 * slot + 1] = -1;
                    prim[3 * slot + 2] = -1;
                    ++leaf_tris;
                } else {
                    st[sp++] = nodes[x].right;
                    st[sp++] = nodes[x].left;
                }
            }
        }
    }
    float* nf = reinterpret_cast<float*>(bytes);
    nf[0] = lo[0];
    nf[1] = lo[1];
    nf[2] = lo[2];
    bytes[12] = (uint8_t)(int8_t)e[0];
    bytes[13] = (uint8_t)(int8_t)e[1];
    bytes[14] = (uint8_t)(int8_t)e[2];
    bytes[15] = imask;
    reinterpret_cast<int32_t*>(bytes)[4] = inner ? (int32_t)base : 0;
    reinterpret_cast<int32_t*>(bytes)[5] = leaf_tris ? (int32_t)tbase : 0;
    for (int q = 0; q < 5; ++q) out_nodes[(int64_t)it.addr * 5 + q] = node[q];
}

unsigned blocks_of(int64_t n, int b) { return (unsigned)std::max<int64_t>(1, (n + b - 1) / b); }

// ---- PLOC: parallel locally-ordered clustering (Meister and Bittner,
// "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
// Construction", IEEE TVCG 2018).  The clusters start as the triangles in
// Morton order; each round every cluster finds, among the kPlocRadius
// clusters on either side of it, the one whose merged box has the least
// surface area, mutual nearest neighbours merge into a new node (placed at
// the lower position), and the array is compacted.  Merged boxes group
// primitives by extent as well as position, which the Morton order alone
// does not.  Node numbers come from prefix sums, counting down from n - 2 in
// position order, so the last merge is the root (node 0) and the tree does
// not depend on thread scheduling.
constexpr int kPlocRadius = 16;

struct CBox {
    float lo[3], hi[3];
};

__device__ inline float merged_area(const CBox& a, const CBox& b) {
    float lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
        lo[q] = fminf(a.lo[q], b.lo[q]);
        hi[q] = fmaxf(a.hi[q], b.hi[q]);
    }
    return half_area(lo, hi);
}

__global__ void ploc_init_kernel(const uint64_t* k, uint64_t idx_mask, int64_t n, const float* v, const int32_t* idx,
                                 int32_t* code, CBox* box) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    code[p] = ~(int32_t)p;
    tri_box(v, idx, key_tri(k, p, idx_mask), box[p].lo, box[p].hi);
}

// Nearest neighbour of each cluster within the radius: least merged area,
// ties to the nearer position, then to the cluster's partner i ^ 1, then to
// the lower position.  The rule is the same seen from both sides of a pair,
// and clusters with identical boxes (duplicated geometry) pair off with
// their partners, half of them merging per round instead of one pair.
__global__ void ploc_nn_kernel(const CBox* box, int64_t m, int32_t* nn) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const CBox bi = box[i];
    const int64_t j0 = i - kPlocRadius < 0 ? 0 : i - kPlocRadius;
    const int64_t j1 = i + kPlocRadius >= m ? m - 1 : i + kPlocRadius;
    float best = FLT_MAX;
    int64_t bj = i == 0 ? 1 : i - 1, bdist = INT64_MAX;
    bool bpartner = false;
    for (int64_t j = j0; j <= j1; ++j) {
        if (j == i) continue;
        const float d = merged_area(bi, box[j]);
        const int64_t dist = j > i ? j - i : i - j;
        const bool partner = j == (i ^ 1);
        // ascending j: among full ties the first is the lowest position
        if (d < best || (d == best && (dist < bdist || (dist == bdist && partner && !bpartner)))) {
            best = d;
            bj = j;
            bdist = dist;
            bpartner = partner;
        }
    }
    nn[i] = (int32_t)bj;
}

// merge[i] = 1 for the lower cluster of a mutual pair; keep[i] = 0 for the
// upper one (it is absorbed).  Both arrays have an extra zero at m for the
// scans' totals.
__global__ void ploc_flags_kernel(const int32_t* nn, int64_t m, int32_t* merge, int32_t* keep) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > m) return;
    if (i == m) {
        merge[i] = 0;
        keep[i] = 0;
        return;
    }
    const int32_t j = nn[i];
    const bool mutual = nn[j] == (int32_t)i;
    merge[i] = mutual && (int32_t)i < j;
    keep[i] = !(mutual && (int32_t)i > j);
}

__global__ void ploc_merge_kernel(const int32_t* nn, const int32_t* merge, const int32_t* rank, int64_t m, int64_t top,
                                  const uint64_t* k, uint64_t idx_mask, const float* v, const int32_t* idx,
                                  int32_t* code, CBox* box, BNode* nodes, int32_t* leaf_parent) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !merge[i]) return;
    const int32_t j = nn[i];
    const int32_t node = (int32_t)(top - rank[i]);
    const int32_t c[2] = {code[i], code[j]};
    float clo[2][3], chi[2][3], cc[2];
    int32_t cn[2];
    for (int q = 0; q < 2; ++q) child_box(nodes, k, idx_mask, v, idx, c[q], clo[q], chi[q], cn[q], &cc[q]);
    BNode& nd = nodes[node];
    nd.left = c[0];
    nd.right = c[1];
    nd.parent = -1;
    nd.count = cn[0] + cn[1];
    CBox u;
    for (int a = 0; a < 3; ++a) {
        u.lo[a] = fminf(clo[0][a], clo[1][a]);
        u.hi[a] = fmaxf(chi[0][a], chi[1][a]);
        nd.lo[a] = u.lo[a];
        nd.hi[a] = u.hi[a];
    }
    nd.cost = node_cost(half_area(u.lo, u.hi), cc[0], cc[1]);
    for (int q = 0; q < 2; ++q) {
        if (c[q] >= 0) nodes[c[q]].parent = node;
        else leaf_parent[~c[q]] = node;
    }
    code[i] = node;
    box[i] = u;
}

__global__ void ploc_compact_kernel(const int32_t* keep, const int32_t* pos, int64_t m, const int32_t* code,
                                    const CBox* box, int32_t* code2, CBox* box2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || !keep[i]) return;
    code2[pos[i]] = code[i];
    box2[pos[i]] = box[i];
}

}  // namespace
}  // namespace rq

using namespace rq;

// PLOC rounds on the clusters of the sorted triangles: nodes, boxes, counts,
// costs and parent links as the radix tree + bottom-up boxes give them.
static rq_status ploc_tree(const uint64_t* keys_sorted, uint64_t idx_mask, int64_t n, const float* vertices,
                           const int32_t* indices, BNode* bn, int32_t* leaf_parent, cudaStream_t s) {
    int32_t *code = nullptr, *code2 = nullptr, *nn = nullptr, *merge = nullptr, *keep = nullptr, *rank = nullptr,
            *pos = nullptr;
    CBox *box = nullptr, *box2 = nullptr;
    void* temp = nullptr;
    size_t temp_bytes = 0;
    rq_status st = RQ_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == RQ_OK) st = cuda_fail(e, "rq_build_scene_gpu (PLOC)");
        return st == RQ_OK;
    };
    const int64_t n1 = n + 1;
    if (ok(cudaMalloc(&code, n * sizeof(int32_t))) && ok(cudaMalloc(&code2, n * sizeof(int32_t))) &&
        ok(cudaMalloc(&nn, n * sizeof(int32_t))) && ok(cudaMalloc(&merge, n1 * sizeof(int32_t))) &&
        ok(cudaMalloc(&keep, n1 * sizeof(int32_t))) && ok(cudaMalloc(&rank, n1 * sizeof(int32_t))) &&
        ok(cudaMalloc(&pos, n1 * sizeof(int32_t))) && ok(cudaMalloc(&box, n * sizeof(CBox))) &&
        ok(cudaMalloc(&box2, n * sizeof(CBox))) &&
        ok(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, merge, rank, (int)n1, s)) &&
        ok(cudaMalloc(&temp, std::max<size_t>(temp_bytes, 1)))) {
        ploc_init_kernel<<<blocks_of(n, 256), 256, 0, s>>>(keys_sorted, idx_mask, n, vertices, indices, code, box);
        ok(cudaGetLastError());
        int64_t m = n, top = n - 2;
        // Each round merges at least the globally closest pair in reach; a
        // round that merges nothing (non-finite boxes) is an error.
        for (int round = 0; st == RQ_OK && m > 1; ++round) {
            if (round > 100000) {
                st = RQ_ERR_BAD_SCENE;
                break;
            }
            ploc_nn_kernel<<<blocks_of(m, 256), 256, 0, s>>>(box, m, nn);
            ploc_flags_kernel<<<blocks_of(m + 1, 256), 256, 0, s>>>(nn, m, merge, keep);
            ok(cudaGetLastError());
            size_t tb = temp_bytes;
            ok(cub::DeviceScan::ExclusiveSum(temp, tb, merge, rank, (int)(m + 1), s));
            tb = temp_bytes;
            ok(cub::DeviceScan::ExclusiveSum(temp, tb, keep, pos, (int)(m + 1), s));
            int32_t totals[2] = {0, 0};
            ok(cudaMemcpyAsync(&totals[0], rank + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            ok(cudaMemcpyAsync(&totals[1], pos + m, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
            ok(cudaStreamSynchronize(s));
            if (st != RQ_OK) break;
            const int64_t merges = totals[0], kept = totals[1];
            if (merges <= 0 || kept != m - merges || top - merges + 1 < 0) {
                st = RQ_ERR_BAD_SCENE;
                break;
            }
            ploc_merge_kernel<<<blocks_of(m, 256), 256, 0, s>>>(nn, merge, rank, m, top, keys_sorted, idx_mask,
                                                                vertices, indices, code, box, bn, leaf_parent);
            ploc_compact_kernel<<<blocks_of(m, 256), 256, 0, s>>>(keep, pos, m, code, box, code2, box2);
            ok(cudaGetLastError());
            std::swap(code, code2);
            std::swap(box, box2);
            top -= merges;
            m = kept;
        }
        if (st == RQ_OK && top != -1) st = RQ_ERR_BAD_SCENE;  // n - 1 nodes, the root last (node 0)
    }
    ok(cudaStreamSynchronize(s));
    cudaFree(code);
    cudaFree(code2);
    cudaFree(nn);
    cudaFree(merge);
    cudaFree(keep);
    cudaFree(rank);
    cudaFree(pos);
    cudaFree(box);
    cudaFree(box2);
    cudaFree(temp);
    return st;
}

// The references of a pre-split mesh: the box mesh (2 corners per
// reference), its index triples and the triangle of each reference.
struct RefMesh {
    float* v = nullptr;
    int32_t* idx = nullptr;
    int32_t* tri = nullptr;
    int64_t n = 0;
    void release() {
        cudaFree(v);
        cudaFree(idx);
        cudaFree(tri);
        *this = RefMesh{};
    }
};

// Cuts the nt triangles into at most nt + nt * budget / 100 references
// (fewer when few triangles waste box area).  Leaves rm.n = 0 when there is
// nothing to split.  The indices have been checked.
static rq_status presplit(const float* v, const int32_t* idx, int64_t nt, int budget, RefMesh& rm, cudaStream_t s) {
    const int64_t extra = std::min<int64_t>((int64_t)((double)nt * budget / 100.0), (int64_t)INT32_MAX / 4 - nt);
    if (extra <= 0) return RQ_OK;
    rq_status st = RQ_OK;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && st == RQ_OK) st = cuda_fail(e, "rq_build_scene_gpu (split)");
        return st == RQ_OK;
    };
    unsigned* sb = nullptr;
    float *prio = nullptr, *sum = nullptr;
    int64_t *pieces = nullptr, *off = nullptr;
    void* temp = nullptr;
    size_t b_sum = 0, b_scan = 0;
    int64_t refs = 0;
    if (ok(cudaMalloc(&sb, 6 * sizeof(unsigned))) && ok(cudaMalloc(&prio, nt * sizeof(float))) &&
        ok(cudaMalloc(&sum, sizeof(float))) && ok(cudaMalloc(&pieces, nt * sizeof(int64_t))) &&
        ok(cudaMalloc(&off, nt * sizeof(int64_t))) &&
        ok(cub::DeviceReduce::Sum(nullptr, b_sum, prio, sum, (int)nt, s)) &&
        ok(cub::DeviceScan::ExclusiveSum(nullptr, b_scan, pieces, off, (int)nt, s)) &&
        ok(cudaMalloc(&temp, std::max<size_t>({b_sum, b_scan, (size_t)1})))) {
        const unsigned init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
        ok(cudaMemcpyAsync(sb, init, sizeof(init), cudaMemcpyHostToDevice, s));
        scene_bounds_kernel<<<std::min<unsigned>(blocks_of(nt, 256), 4 * 148), 256, 0, s>>>(v, idx, nt, sb);
        split_priority_kernel<<<blocks_of(nt, 256), 256, 0, s>>>(v, idx, nt, sb, prio);
        ok(cudaGetLastError());
        ok(cub::DeviceReduce::Sum(temp, b_sum, prio, sum, (int)nt, s));
        split_count_kernel<<<blocks_of(nt, 256), 256, 0, s>>>(prio, nt, sum, (double)extra, pieces);
        ok(cudaGetLastError());
        ok(cub::DeviceScan::ExclusiveSum(temp, b_scan, pieces, off, (int)nt, s));
        int64_t tail[2] = {0, 0};
        ok(cudaMemcpyAsync(&tail[0], off + nt - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        ok(cudaMemcpyAsync(&tail[1], pieces + nt - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        ok(cudaStreamSynchronize(s));
        refs = tail[0] + tail[1];
        if (st == RQ_OK && (refs < nt || refs > (int64_t)INT32_MAX / 4)) st = RQ_ERR_INVALID_ARG;
    }
    if (st == RQ_OK && refs > nt) {
        if (ok(cudaMalloc(&rm.v, refs * 6 * sizeof(float))) && ok(cudaMalloc(&rm.idx, refs * 3 * sizeof(int32_t))) &&
            ok(cudaMalloc(&rm.tri, refs * sizeof(int32_t)))) {
            split_kernel<<<blocks_of(nt, 128), 128, 0, s>>>(v, idx, nt, sb, pieces, off, rm.v, rm.idx, rm.tri);
            ok(cudaGetLastError());
            rm.n = refs;
        }
    }
    if (st != RQ_OK) rm.release();
    ok(cudaStreamSynchronize(s));  // the temporaries below are freed after the kernels that read them
    cudaFree(sb);
    cudaFree(prio);
    cudaFree(sum);
    cudaFree(pieces);
    cudaFree(off);
    cudaFree(temp);
    return st;
}

extern "C" rq_status rq_build_scene_gpu(const float* vertices, int64_t nv, const int32_t* indices, int64_t nt,
                                        int method, int optimize_passes, int split_budget, rq_scene_t* out,
                                        void* stream) {
    if (!out || !vertices || !indices || nv <= 0 || nt <= 0 || nt > (int64_t)INT32_MAX / 4) return RQ_ERR_INVALID_ARG;
    const bool thread_treelets = (method & RQ_GPU_BUILD_THREAD_TREELETS) != 0;
    method &= ~RQ_GPU_BUILD_THREAD_TREELETS;
    if (method != RQ_GPU_BUILD_LBVH && method != RQ_GPU_BUILD_PLOC) return RQ_ERR_INVALID_ARG;
    if (split_budget < 0 || split_budget > 400) return RQ_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    {
        // indices first: every kernel below reads vertices through them
        unsigned* bad_d = nullptr;
        unsigned bad = 0;
        RQ_CUDA(cudaMalloc(&bad_d, sizeof(unsigned)));
        cudaError_t e = cudaMemsetAsync(bad_d, 0, sizeof(unsigned), s);
        if (e == cudaSuccess) {
            check_indices_kernel<<<std::min<unsigned>(blocks_of(3 * nt, 256), 8 * 148), 256, 0, s>>>(
                indices, 3 * nt, nv, bad_d);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, bad_d, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(bad_d);
        if (e != cudaSuccess) return cuda_fail(e, "rq_build_scene_gpu");
        if (bad) return RQ_ERR_INVALID_ARG;
    }
    RefMesh rm;
    if (split_budget > 0) {
        const rq_status ps = presplit(vertices, indices, nt, split_budget, rm, s);
        if (ps != RQ_OK) return ps;
    }
    // The tree stages read boxes from the box mesh when the triangles were
    // split, from the triangles otherwise; leaves map back through rm.tri.
    const float* bv = rm.n ? rm.v : vertices;
    const int32_t* bi = rm.n ? rm.idx : indices;
    const int64_t n = rm.n ? rm.n : nt;
    // device scratch
    uint64_t *keys = nullptr, *keys_sorted = nullptr;
    BNode* bn = nullptr;
    int32_t *leaf_parent = nullptr, *arrivals = nullptr;
    CollapseDP* dp = nullptr;
    unsigned* ob = nullptr;
    Item *qa = nullptr, *qb = nullptr;
    Ctr* ctr = nullptr;
    void* cub_temp = nullptr;
    float4 *nodes = nullptr, *woop = nullptr;
    int32_t* prim = nullptr;
    size_t cub_bytes = 0;
    int idx_bits = 1;
    while ((1ll << idx_bits) < n) ++idx_bits;
    const uint64_t idx_mask = (1ull << idx_bits) - 1;
    const int axis_bits = std::min(21, (64 - idx_bits) / 3);
    const int end_bit = idx_bits + 3 * axis_bits;
    rq_status st = RQ_OK;
    auto ok = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess && st == RQ_OK) st = cuda_fail(e, what);
        return st == RQ_OK;
    };
    const int64_t node_cap = std::max<int64_t>(1, n);  // an 8-wide node per binary node at most
    const int64_t q_cap = node_cap;
    constexpr size_t kPad = 256;
    if (ok(cudaMalloc(&keys, n * sizeof(uint64_t)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&keys_sorted, n * sizeof(uint64_t)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&bn, std::max<int64_t>(1, n - 1) * sizeof(BNode)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&leaf_parent, n * sizeof(int32_t)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&arrivals, std::max<int64_t>(1, n - 1) * sizeof(int32_t)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&dp, std::max<int64_t>(1, n - 1) * sizeof(CollapseDP)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&ob, 6 * sizeof(unsigned)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&qa, q_cap * sizeof(Item)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&qb, q_cap * sizeof(Item)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&ctr, sizeof(Ctr)), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&nodes, node_cap * 80 + kPad), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&woop, n * 48 + kPad), "rq_build_scene_gpu") &&
        ok(cudaMalloc(&prim, n * 12), "rq_build_scene_gpu")) {
        const unsigned init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
        ok(cudaMemcpyAsync(ob, init, sizeof(init), cudaMemcpyHostToDevice, s), "rq_build_scene_gpu");
        ok(cudaMemsetAsync(nodes, 0, node_cap * 80 + kPad, s), "rq_build_scene_gpu");
        ok(cudaMemsetAsync(woop, 0, n * 48 + kPad, s), "rq_build_scene_gpu");
        ok(cudaMemsetAsync(arrivals, 0, std::max<int64_t>(1, n - 1) * sizeof(int32_t), s), "rq_build_scene_gpu");
        ok(cudaMemsetAsync(ctr, 0, sizeof(Ctr), s), "rq_build_scene_gpu");
    }
    if (st == RQ_OK) {
        centroid_bounds_kernel<<<std::min<unsigned>(blocks_of(n, 256), 4 * 148), 256, 0, s>>>(bv, bi, n, ob);
        morton_kernel<<<blocks_of(n, 256), 256, 0, s>>>(bv, bi, n, ob, axis_bits, idx_bits, keys);
        ok(cudaGetLastError(), "rq_build_scene_gpu");
        ok(cub::DeviceRadixSort::SortKeys(nullptr, cub_bytes, keys, keys_sorted, (int)n, 0, end_bit, s),
           "rq_build_scene_gpu");
        ok(cudaMalloc(&cub_temp, std::max<size_t>(cub_bytes, 1)), "rq_build_scene_gpu");
        ok(cub::DeviceRadixSort::SortKeys(cub_temp, cub_bytes, keys, keys_sorted, (int)n, 0, end_bit, s),
           "rq_build_scene_gpu");
    }
    int64_t levels = 0, n_nodes = 1;
    if (st == RQ_OK && n > 1) {
        if (method == RQ_GPU_BUILD_PLOC) {
            st = ploc_tree(keys_sorted, idx_mask, n, bv, bi, bn, leaf_parent, s);
        } else {
            radix_tree_kernel<<<blocks_of(n - 1, 256), 256, 0, s>>>(keys_sorted, n, bn, leaf_parent);
            boxes_kernel<<<blocks_of(n, 256), 256, 0, s>>>(keys_sorted, idx_mask, n, bv, bi, bn,
                                                           leaf_parent, arrivals);
            ok(cudaGetLastError(), "rq_build_scene_gpu");
        }
        for (int pass = 0; pass < optimize_passes && st == RQ_OK; ++pass) {
            ok(cudaMemsetAsync(arrivals, 0, (n - 1) * sizeof(int32_t), s), "rq_build_scene_gpu");
            if (thread_treelets)
                treelet_kernel<<<blocks_of(n, 128), 128, 0, s>>>(keys_sorted, idx_mask, n, bv, bi, bn,
                                                                 leaf_parent, arrivals, kTreeletLeaves);
            else
                treelet_warp_kernel<<<blocks_of(n, kTreeletWarpBlock), kTreeletWarpBlock, 0, s>>>(
                    keys_sorted, idx_mask, n, bv, bi, bn, leaf_parent, arrivals, kTreeletLeaves);
            ok(cudaGetLastError(), "rq_build_scene_gpu");
        }
        if (st == RQ_OK) {
            ok(cudaMemsetAsync(arrivals, 0, (n - 1) * sizeof(int32_t), s), "rq_build_scene_gpu");
            collapse_dp_kernel<<<blocks_of(n, 256), 256, 0, s>>>(keys_sorted, idx_mask, n, bv, bi, bn,
                                                                 leaf_parent, arrivals, dp);
            ok(cudaGetLastError(), "rq_build_scene_gpu");
        }
    }
    if (st == RQ_OK) {
        // level 0: the root (binary node 0, or the single triangle)
        const Item root{n > 1 ? 0 : ~0, 0};
        const Ctr c0{1ull, 0ull, 0ull, 0u};
        ok(cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, s), "rq_build_scene_gpu");
        ok(cudaMemcpyAsync(ctr, &c0, sizeof(c0), cudaMemcpyHostToDevice, s), "rq_build_scene_gpu");
        int64_t n_items = 1;
        while (st == RQ_OK && n_items > 0) {
            expand_kernel<<<blocks_of(n_items, 128), 128, 0, s>>>(qa, n_items, qb, q_cap, bn, keys_sorted, idx_mask,
                                                                  bv, bi, vertices, indices, rm.tri, nodes, node_cap,
                                                                  woop, prim, n,
                                                                  ctr, n > 1 ? dp : nullptr);
            ok(cudaGetLastError(), "rq_build_scene_gpu");
            Ctr c{};
            ok(cudaMemcpyAsync(&c, ctr, sizeof(Ctr), cudaMemcpyDeviceToHost, s), "rq_build_scene_gpu");
            ok(cudaStreamSynchronize(s), "rq_build_scene_gpu");
            if (st != RQ_OK) break;
            if (c.error) {
                st = RQ_ERR_BAD_SCENE;  // capacity exceeded: cannot happen for a valid radix tree
                break;
            }
            n_items = (int64_t)c.next;
            n_nodes = (int64_t)c.nodes;
            std::swap(qa, qb);
            ok(cudaMemsetAsync(&ctr->next, 0, sizeof(unsigned long long), s), "rq_build_scene_gpu");
            if (++levels > 4096) st = RQ_ERR_BAD_SCENE;
        }
    }
    float root[20] = {};
    if (st == RQ_OK) ok(cudaMemcpy(root, nodes, sizeof(root), cudaMemcpyDeviceToHost), "rq_build_scene_gpu");
    cudaFree(keys);
    cudaFree(keys_sorted);
    cudaFree(bn);
    cudaFree(leaf_parent);
    cudaFree(arrivals);
    cudaFree(dp);
    cudaFree(ob);
    cudaFree(qa);
    cudaFree(qb);
    cudaFree(ctr);
    cudaFree(cub_temp);
    rm.release();
    if (st != RQ_OK) {
        cudaFree(nodes);
        cudaFree(woop);
        cudaFree(prim);
        return st;
    }
    rq_scene* sc = new rq_scene();
    sc->kind = RQ_BVH_CWBVH;
    cudaGetDevice(&sc->device);
    sc->nodes = nodes;
    sc->woop = woop;
    sc->prim_index = prim;
    sc->node_f4 = n_nodes * 5;
    sc->woop_f4 = n * 3;
    sc->prim_count = n * 3;
    sc->owned = true;
    uint32_t ew;
    std::memcpy(&ew, &root[3], 4);
    for (int a = 0; a < 3; ++a) {
        const int e = (int)(int8_t)((ew >> (8 * a)) & 0xFFu);
        sc->lo[a] = root[a];
        sc->hi[a] = root[a] + 255.0f * std::ldexp(1.0f, e);
    }
    *out = sc;
    return RQ_OK;
}
