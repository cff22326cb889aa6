// Binned-SAH BVH builder.  It stands in for the reference's Embree build
// (BuildBVH2Triangle / BuildBVH8Triangle, src/EmbreeBVHBuilder.cpp:303-478),
// which is not available here.  A binary tree is built top-down with a binned
// surface-area heuristic: object splits, and binned spatial splits that
// reference a triangle from both sides within a duplicate budget (200 % of the
// triangle count by default), as Embree's high-quality builder does.  SAH
// treelet restructuring then improves the binary tree, and the 8-wide tree for
// the CWBVH is made by collapsing it with a surface-area cost model (see
// collapse_optimal).  Leaves of the 8-wide tree hold at most 3
// triangles, as the reference asks Embree for (maxLeafSize = 3,
// src/EmbreeBVHBuilder.cpp:456-457).
//
// Speed: primitive records (box + id, 32 B) are moved by the partition, so
// every pass is sequential; one pass bins all three axes and records each
// bin's box and centroid box, from which the children's bounds follow without
// another pass; subtrees above a size threshold are built on other threads.
#include <algorithm>
#include <array>
#include <atomic>
#include <future>
#include <thread>

#include "host_common.h"

namespace rq {
namespace {

constexpr int kMaxBins = 64;
constexpr float kTraversalCost = 1.0f;
constexpr float kIntersectCost = 1.0f;
constexpr int64_t kParallelGrain = 32768;

struct alignas(32) PrimRef {
    float lo[3];
    int32_t id;
    float hi[3];
    int32_t pad;
};

// Plain min/max (inputs are finite); compiles to minss/maxss.
inline float fmn(float a, float b) { return a < b ? a : b; }
inline float fmx(float a, float b) { return a > b ? a : b; }

struct BBox {
    float lo[3] = {INFINITY, INFINITY, INFINITY};
    float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    void grow(const float* l, const float* h) {
        for (int a = 0; a < 3; ++a) { lo[a] = fmn(lo[a], l[a]); hi[a] = fmx(hi[a], h[a]); }
    }
    void grow_pt(const float* p) { grow(p, p); }
    void grow(const BBox& b) { grow(b.lo, b.hi); }
    float area() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0.f && dy >= 0.f && dz >= 0.f)) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
};

struct Bin {
    BBox box, cbox;
    int count = 0;
};

inline void centroid(const PrimRef& p, float c[3]) {
    for (int a = 0; a < 3; ++a) c[a] = (p.lo[a] + p.hi[a]) * 0.5f;
}

// Box of the part of triangle `tri` (vertices v[0..2]) that lies in the slab
// lo <= x[axis] <= hi, intersected with `clip`.  Edge/plane intersections are
// computed in double and rounded outwards, so the box contains the exact
// part; false when the part is empty.
bool slab_box(const float (*v)[3], int axis, float lo, float hi, const BBox& clip, BBox& out) {
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    bool any = false;
    auto grow = [&](const double* q) {
        for (int a = 0; a < 3; ++a) { mn[a] = std::min(mn[a], q[a]); mx[a] = std::max(mx[a], q[a]); }
        any = true;
    };
    for (int e = 0; e < 3; ++e) {
        const float* p = v[e];
        const float* q = v[(e + 1) % 3];
        if (p[axis] >= lo && p[axis] <= hi) {
            const double d[3] = {p[0], p[1], p[2]};
            grow(d);
        }
        for (const float plane : {lo, hi}) {
            if (!std::isfinite(plane)) continue;
            const double dp = (double)p[axis] - plane, dq = (double)q[axis] - plane;
            if (!((dp < 0.0 && dq > 0.0) || (dp > 0.0 && dq < 0.0))) continue;
            const double t = dp / (dp - dq);
            double x[3];
            for (int a = 0; a < 3; ++a) x[a] = (double)p[a] + t * ((double)q[a] - (double)p[a]);
            x[axis] = plane;
            grow(x);
        }
    }
    if (!any) return false;
    for (int a = 0; a < 3; ++a) {
        float l = (float)mn[a], h = (float)mx[a];
        if ((double)l > mn[a]) l = std::nextafter(l, -INFINITY);
        if ((double)h < mx[a]) h = std::nextafter(h, INFINITY);
        if (a == axis) { l = fmx(l, lo); h = fmn(h, hi); }
        out.lo[a] = fmx(l, clip.lo[a]);
        out.hi[a] = fmn(h, clip.hi[a]);
        if (out.lo[a] > out.hi[a]) return false;
    }
    return true;
}

struct Builder2 {
    int max_leaf, bins, max_depth;
    bool big_leaves;  // at the depth cap: one oversized leaf (BVH2) or median splits (CWBVH source)
    // Spatial splits (Stich, Friedrich and Dietrich, "Spatial Splits in
    // Bounding Volume Hierarchies", HPG 2009) need the triangles; they are
    // tried where the object split's children overlap by more than
    // split_alpha of the root's area.
    const Mesh* mesh = nullptr;
    float split_alpha = 1e-5f;
    float root_area = 0.f;
    int spatial_bins = 8;
    int64_t spatial_min = 0;  // nodes with fewer references use object splits only
    // refs[begin, end) are a node's references and refs[end, cap) the slack
    // its subtree may fill with spatial-split duplicates; slack is handed to
    // the children in proportion to their sizes, so the tree does not depend
    // on the order in which subtrees are built.
    std::vector<PrimRef> refs;
    std::vector<TreeNode<2>> nodes;
    std::vector<Leaf> leaves;
    std::atomic<int32_t> n_nodes{0};
    std::atomic<int32_t> n_leaves{0};
    std::atomic<int> spare_threads{0};

    struct Range {
        int64_t begin, end, cap;
        BBox box, cbox;
    };

    // Threads for binning one large node; nodes below kParallelBin
    // references are binned by the thread that builds them.
    int threads_total = 1;
    static constexpr int64_t kParallelBin = int64_t(1) << 20;
    int64_t chunks_for(int64_t n) const {
        if (threads_total <= 1 || n < kParallelBin) return 1;
        return std::min<int64_t>(threads_total, n / (kParallelBin / 4));
    }

    int32_t make_leaf(int64_t begin, int64_t end) {
        // Fragments of one split triangle can share a leaf: keep one of each.
        int64_t n = 0;
        for (int64_t k = begin; k < end; ++k) {
            bool dup = false;
            for (int64_t j = begin; j < begin + n; ++j) dup = dup || refs[j].id == refs[k].id;
            if (!dup) refs[begin + n++] = refs[k];
        }
        const int32_t l = n_leaves.fetch_add(1);
        leaves[l] = Leaf{(int32_t)begin, (int32_t)n};
        return -(l + 2);
    }

    void tri_verts(int32_t id, float v[3][3]) const {
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) v[k][a] = mesh->v[3 * (size_t)mesh->i[3 * (int64_t)id + k] + a];
    }

    // Bounds of refs[begin, end) and of their centroids.
    void bounds_of(int64_t begin, int64_t end, BBox& b, BBox& cb) const {
        b = BBox();
        cb = BBox();
        for (int64_t k = begin; k < end; ++k) {
            float c[3];
            centroid(refs[k], c);
            b.grow(refs[k].lo, refs[k].hi);
            cb.grow_pt(c);
        }
    }

    // Splits the slack of [begin, cap) between children of nl and nr
    // references placed at begin: returns the left child's slack.
    static int64_t left_slack(int64_t slack, int64_t nl, int64_t nr) {
        return slack <= 0 ? 0 : (int64_t)((__int128)slack * nl / (nl + nr));
    }

    // Child code of the subtree over refs[begin, end) with slack up to cap,
    // bounds `b` and centroid bounds `cb`.
    int32_t build(int64_t begin, int64_t end, int64_t cap, const BBox& b, const BBox& cb, int depth) {
        const int64_t n = end - begin;
        const bool may_leaf = n <= max_leaf;
        if (n == 1 || (depth >= max_depth && (may_leaf || big_leaves))) return make_leaf(begin, end);
        if (depth >= max_depth) return median_split(begin, end, cap, cb, depth);

        // One pass: bin all three axes (fewer bins for small nodes: the bin
        // arrays are initialised per node).
        const int nb = (int)std::min<int64_t>(bins, std::max<int64_t>(4, n));
        float scale[3];
        bool usable[3];
        for (int a = 0; a < 3; ++a) {
            const float ext = cb.hi[a] - cb.lo[a];
            usable[a] = ext > 0.f;
            scale[a] = usable[a] ? (float)nb / ext : 0.f;
        }
        alignas(Bin) unsigned char storage[3 * kMaxBins * sizeof(Bin)];
        Bin(*bin)[kMaxBins] = reinterpret_cast<Bin(*)[kMaxBins]>(storage);
        for (int a = 0; a < 3; ++a)
            for (int i = 0; i < nb; ++i) new (&bin[a][i]) Bin();
        auto bin_refs = [&](int64_t k0, int64_t k1, Bin (*out)[kMaxBins]) {
            for (int64_t k = k0; k < k1; ++k) {
                const PrimRef& p = refs[k];
                float c[3];
                centroid(p, c);
                for (int a = 0; a < 3; ++a) {
                    int bi = (int)((c[a] - cb.lo[a]) * scale[a]);
                    bi = bi < 0 ? 0 : (bi >= nb ? nb - 1 : bi);
                    Bin& x = out[a][bi];
                    x.count++;
                    x.box.grow(p.lo, p.hi);
                    x.cbox.grow_pt(c);
                }
            }
        };
        const int64_t chunks = chunks_for(n);
        if (chunks <= 1) {
            bin_refs(begin, end, bin);
        } else {
            // Large nodes (the top of the tree, built before the subtrees
            // spread over the threads): bin chunks in parallel, then merge;
            // min/max and counts do not depend on the order.
            std::vector<std::array<std::array<Bin, kMaxBins>, 3>> part((size_t)chunks);
            parallel_tasks(chunks, threads_total, [&](int64_t c) {
                Bin(*out)[kMaxBins] = reinterpret_cast<Bin(*)[kMaxBins]>(part[(size_t)c].data());
                bin_refs(begin + n * c / chunks, begin + n * (c + 1) / chunks, out);
            });
            for (const auto& pc : part)
                for (int a = 0; a < 3; ++a)
                    for (int i = 0; i < nb; ++i) {
                        bin[a][i].count += pc[(size_t)a][(size_t)i].count;
                        bin[a][i].box.grow(pc[(size_t)a][(size_t)i].box);
                        bin[a][i].cbox.grow(pc[(size_t)a][(size_t)i].cbox);
                    }
        }
        float best_cost = INFINITY;
        int best_axis = -1, best_bin = -1;
        for (int a = 0; a < 3; ++a) {
            if (!usable[a]) continue;
            float right_area[kMaxBins];
            int right_count[kMaxBins];
            BBox rb;
            int rc = 0;
            for (int i = nb - 1; i > 0; --i) {
                rb.grow(bin[a][i].box);
                rc += bin[a][i].count;
                right_area[i] = rb.area();
                right_count[i] = rc;
            }
            BBox lb;
            int lc = 0;
            for (int i = 0; i < nb - 1; ++i) {
                lb.grow(bin[a][i].box);
                lc += bin[a][i].count;
                if (lc == 0 || right_count[i + 1] == 0) continue;
                const float c = lb.area() * lc + right_area[i + 1] * right_count[i + 1];
                if (c < best_cost) { best_cost = c; best_axis = a; best_bin = i; }
            }
        }
        const float parent_area = b.area();
        const float split_cost =
            kTraversalCost + kIntersectCost * (parent_area > 0.f ? best_cost / parent_area : 0.f);
        if (may_leaf && (best_axis < 0 || kIntersectCost * (float)n <= split_cost)) return make_leaf(begin, end);

        BBox lb, lcb, rb, rcb;
        if (best_axis >= 0) {
            for (int i = 0; i < nb; ++i) {
                if (i <= best_bin) { lb.grow(bin[best_axis][i].box); lcb.grow(bin[best_axis][i].cbox); }
                else { rb.grow(bin[best_axis][i].box); rcb.grow(bin[best_axis][i].cbox); }
            }
        }
        int32_t code;
        if (mesh && cap > end && try_spatial(begin, end, cap, b, best_axis >= 0 ? best_cost : INFINITY, lb, rb,
                                             depth, best_axis >= 0, code))
            return code;
        if (best_axis < 0) return median_split(begin, end, cap, cb, depth);  // all centroids coincide

        const int a = best_axis;
        const float lo = cb.lo[a], sc = scale[a];
        PrimRef* first = refs.data() + begin;
        PrimRef* m = std::partition(first, refs.data() + end, [&](const PrimRef& p) {
            int bi = (int)(((p.lo[a] + p.hi[a]) * 0.5f - lo) * sc);
            bi = bi < 0 ? 0 : (bi >= nb ? nb - 1 : bi);
            return bi <= best_bin;
        });
        const int64_t mid = begin + (m - first);
        if (mid == begin || mid == end) return median_split(begin, end, cap, cb, depth);
        return object_children(begin, mid, end, cap, lb, lcb, rb, rcb, depth);
    }

    // Children [begin, mid) and [mid, end) of an in-place partition; the
    // right block moves up by the left child's slack.
    int32_t object_children(int64_t begin, int64_t mid, int64_t end, int64_t cap, const BBox& lb, const BBox& lcb,
                            const BBox& rb, const BBox& rcb, int depth) {
        const int64_t sl = left_slack(cap - end, mid - begin, end - mid);
        if (sl > 0) std::move_backward(refs.data() + mid, refs.data() + end, refs.data() + end + sl);
        return make_inner(Range{begin, mid, mid + sl, lb, lcb}, Range{mid + sl, end + sl, cap, rb, rcb}, depth);
    }

    // Binned spatial split of refs[begin, end) (bins over the node's box);
    // taken, with reference unsplitting, when cheaper than the object split
    // and within the slack.  On success the node is built and its code
    // returned in `code`.
    bool try_spatial(int64_t begin, int64_t end, int64_t cap, const BBox& b, float object_cost, const BBox& olb,
                     const BBox& orb, int depth, bool have_object, int32_t& code) {
        const int64_t n = end - begin;
        if (n < spatial_min) return false;
        if (have_object) {
            BBox ov;
            for (int a = 0; a < 3; ++a) { ov.lo[a] = fmx(olb.lo[a], orb.lo[a]); ov.hi[a] = fmn(olb.hi[a], orb.hi[a]); }
            if (!(ov.area() > split_alpha * root_area)) return false;
        }
        const int nb = (int)std::min<int64_t>(spatial_bins, std::max<int64_t>(4, n));
        struct SBin {
            BBox box;
            int enter = 0, exit = 0;
        };
        float best = object_cost;
        int best_axis = -1, best_plane = -1;
        int64_t best_nl = 0, best_nr = 0;
        // Plane k of axis a (k = 0..nb); bin j lies between planes j and j+1.
        float planes[3][kMaxBins + 1], to_bin[3];
        for (int a = 0; a < 3; ++a) {
            const float ext = b.hi[a] - b.lo[a];
            for (int k = 0; k <= nb; ++k)
                planes[a][k] = k == 0 ? b.lo[a] : (k == nb ? b.hi[a] : b.lo[a] + ext * ((float)k / (float)nb));
            to_bin[a] = ext > 0.f ? (float)nb / ext : 0.f;
        }
        auto plane = [&](int ax, int k) { return planes[ax][k]; };
        auto bin_of = [&](int a, float x) {
            int k = (int)((x - b.lo[a]) * to_bin[a]);
            k = k < 0 ? 0 : (k >= nb ? nb - 1 : k);
            while (k > 0 && x < planes[a][k]) --k;
            while (k < nb - 1 && x >= planes[a][k + 1]) ++k;
            return k;
        };
        SBin sbin[3][kMaxBins];
        bool usable[3];
        for (int a = 0; a < 3; ++a) usable[a] = b.hi[a] - b.lo[a] > 0.f;
        auto bin_refs = [&](int64_t k0, int64_t k1, SBin (*out)[kMaxBins]) {
            for (int64_t k = k0; k < k1; ++k) {
                const PrimRef& r = refs[k];
                BBox rbox;
                rbox.grow(r.lo, r.hi);
                for (int a = 0; a < 3; ++a) {
                    if (!usable[a]) continue;
                    const int b0 = bin_of(a, r.lo[a]), b1 = bin_of(a, r.hi[a]);
                    out[a][b0].enter++;
                    out[a][b1].exit++;
                    for (int j = b0; j <= b1; ++j) {
                        BBox q = rbox;
                        q.lo[a] = fmx(q.lo[a], plane(a, j));
                        q.hi[a] = fmn(q.hi[a], plane(a, j + 1));
                        out[a][j].box.grow(q);
                    }
                }
            }
        };
        const int64_t chunks = chunks_for(n);
        if (chunks <= 1) {
            bin_refs(begin, end, sbin);
        } else {
            std::vector<std::array<std::array<SBin, kMaxBins>, 3>> part((size_t)chunks);
            parallel_tasks(chunks, threads_total, [&](int64_t c) {
                SBin(*out)[kMaxBins] = reinterpret_cast<SBin(*)[kMaxBins]>(part[(size_t)c].data());
                bin_refs(begin + n * c / chunks, begin + n * (c + 1) / chunks, out);
            });
            for (const auto& pc : part)
                for (int a = 0; a < 3; ++a)
                    for (int i = 0; i < nb; ++i) {
                        sbin[a][i].enter += pc[(size_t)a][(size_t)i].enter;
                        sbin[a][i].exit += pc[(size_t)a][(size_t)i].exit;
                        sbin[a][i].box.grow(pc[(size_t)a][(size_t)i].box);
                    }
        }
        for (int a = 0; a < 3; ++a) {
            if (!usable[a]) continue;
            const SBin* sb = sbin[a];
            float right_area[kMaxBins];
            int64_t right_count[kMaxBins];
            BBox rb;
            int64_t rc = 0;
            for (int i = nb - 1; i > 0; --i) {
                rb.grow(sb[i].box);
                rc += sb[i].exit;
                right_area[i] = rb.area();
                right_count[i] = rc;
            }
            BBox lb;
            int64_t lc = 0;
            for (int i = 0; i < nb - 1; ++i) {
                lb.grow(sb[i].box);
                lc += sb[i].enter;
                const int64_t nr = right_count[i + 1];
                if (lc == 0 || nr == 0 || lc == n || nr == n) continue;
                if (begin + lc + nr > cap) continue;  // over this subtree's budget
                const float c = lb.area() * (float)lc + right_area[i + 1] * (float)nr;
                if (c < best) { best = c; best_axis = a; best_plane = i + 1; best_nl = lc; best_nr = nr; }
            }
        }
        if (best_axis < 0) return false;

        // Distribute: wholly left / right, or straddling (split or unsplit).
        const int a = best_axis;
        const float pos = planes[a][best_plane];
        std::vector<PrimRef> left, right, straddle;
        left.reserve((size_t)best_nl);
        right.reserve((size_t)best_nr);
        BBox lbox, rbox;
        for (int64_t k = begin; k < end; ++k) {
            const PrimRef& r = refs[k];
            if (r.hi[a] <= pos) { left.push_back(r); lbox.grow(r.lo, r.hi); }
            else if (r.lo[a] >= pos) { right.push_back(r); rbox.grow(r.lo, r.hi); }
            else straddle.push_back(r);
        }
        for (size_t si = 0; si < straddle.size(); ++si) {
            const PrimRef& r = straddle[si];
            const int64_t still = (int64_t)(straddle.size() - si - 1);  // each takes >= 1 slot
            BBox whole;
            whole.grow(r.lo, r.hi);
            float v[3][3];
            tri_verts(r.id, v);
            BBox lp, rp;
            const bool hl = slab_box(v, a, -INFINITY, pos, whole, lp);
            const bool hr = slab_box(v, a, pos, INFINITY, whole, rp);
            const float nl = (float)left.size(), nr = (float)right.size();
            BBox l_all = lbox, r_all = rbox;
            l_all.grow(whole);
            r_all.grow(whole);
            BBox l_split = lbox, r_split = rbox;
            if (hl) l_split.grow(lp);
            if (hr) r_split.grow(rp);
            const float c_split = hl && hr ? l_split.area() * (nl + 1) + r_split.area() * (nr + 1) : INFINITY;
            const float c_left = l_all.area() * (nl + 1) + rbox.area() * nr;
            const float c_right = lbox.area() * nl + r_all.area() * (nr + 1);
            if (c_split < c_left && c_split < c_right &&
                begin + (int64_t)left.size() + (int64_t)right.size() + 2 + still <= cap) {
                PrimRef pl = r, pr = r;
                for (int q = 0; q < 3; ++q) {
                    pl.lo[q] = lp.lo[q]; pl.hi[q] = lp.hi[q];
                    pr.lo[q] = rp.lo[q]; pr.hi[q] = rp.hi[q];
                }
                left.push_back(pl);
                right.push_back(pr);
                lbox.grow(lp);
                rbox.grow(rp);
            } else if (c_left <= c_right) {
                left.push_back(r);
                lbox.grow(whole);
            } else {
                right.push_back(r);
                rbox.grow(whole);
            }
        }
        const int64_t nl = (int64_t)left.size(), nr = (int64_t)right.size();
        // Unsplitting emptied a side or kept every reference on one side:
        // the node is left to the object split.
        if (nl == 0 || nr == 0 || nl == n || nr == n || begin + nl + nr > cap) return false;
        const int64_t sl = left_slack(cap - begin - nl - nr, nl, nr);
        std::copy(left.begin(), left.end(), refs.data() + begin);
        std::copy(right.begin(), right.end(), refs.data() + begin + nl + sl);
        BBox lb, lcb, rb, rcb;
        bounds_of(begin, begin + nl, lb, lcb);
        bounds_of(begin + nl + sl, begin + nl + sl + nr, rb, rcb);
        code = make_inner(Range{begin, begin + nl, begin + nl + sl, lb, lcb},
                          Range{begin + nl + sl, begin + nl + sl + nr, cap, rb, rcb}, depth);
        return true;
    }

    // Balanced split at the centroid median of the widest centroid axis; keeps
    // the depth bounded by log2(n) once the SAH recursion reaches the cap.
    int32_t median_split(int64_t begin, int64_t end, int64_t cap, const BBox& cb, int depth) {
        int axis = 0;
        float widest = -1.f;
        for (int a = 0; a < 3; ++a)
            if (cb.hi[a] - cb.lo[a] > widest) { widest = cb.hi[a] - cb.lo[a]; axis = a; }
        const int64_t mid = begin + (end - begin) / 2;
        std::nth_element(refs.data() + begin, refs.data() + mid, refs.data() + end,
                         [&](const PrimRef& x, const PrimRef& y) {
                             return x.lo[axis] + x.hi[axis] < y.lo[axis] + y.hi[axis];
                         });
        BBox lb, lcb, rb, rcb;
        bounds_of(begin, mid, lb, lcb);
        bounds_of(mid, end, rb, rcb);
        return object_children(begin, mid, end, cap, lb, lcb, rb, rcb, depth);
    }

    int32_t make_inner(const Range& l, const Range& r, int depth) {
        const int64_t n = (l.end - l.begin) + (r.end - r.begin);
        const int32_t me = n_nodes.fetch_add(1);
        int32_t lc, rc;
        bool spawned = false;
        std::future<int32_t> fut;
        if (n > kParallelGrain) {
            if (spare_threads.fetch_sub(1) > 0) {
                spawned = true;
                fut = std::async(std::launch::async,
                                 [=, this] { return build(l.begin, l.end, l.cap, l.box, l.cbox, depth + 1); });
            } else {
                spare_threads.fetch_add(1);
            }
        }
        if (spawned) {
            rc = build(r.begin, r.end, r.cap, r.box, r.cbox, depth + 1);
            lc = fut.get();
            spare_threads.fetch_add(1);
        } else {
            lc = build(l.begin, l.end, l.cap, l.box, l.cbox, depth + 1);
            rc = build(r.begin, r.end, r.cap, r.box, r.cbox, depth + 1);
        }
        TreeNode<2> node{};
        node.count = 2;
        node.child[0] = lc;
        node.child[1] = rc;
        for (int a = 0; a < 3; ++a) {
            node.lo[0][a] = l.box.lo[a]; node.hi[0][a] = l.box.hi[a];
            node.lo[1][a] = r.box.lo[a]; node.hi[1][a] = r.box.hi[a];
        }
        nodes[me] = node;
        return me;
    }
};

}  // namespace

// ----------------------------------------------------------- pre-splitting --
// A long thin triangle lying diagonally in its box (common in steep terrain)
// has a box far larger than itself, and rays entering the box mostly miss
// it.  Before the build such triangles are cut at the midplane of their box's
// longest axis, recursively, into up to `max_frags` fragments; each fragment
// is a reference to the same triangle with the bounds of the clipped polygon.
// Triangles are taken worst fit first (box area / triangle area) until one
// extra reference per triangle has been spent.  Leaves keep one reference per
// triangle, so results are unchanged; only boxes get tighter.
namespace {

// Sutherland-Hodgman clip of a convex polygon to x[axis] <= pos (below) or
// >= pos (above).
int clip_polygon(const float (*in)[3], int n, int axis, float pos, bool below, float (*out)[3]) {
    int m = 0;
    for (int i = 0; i < n; ++i) {
        const float* a = in[i];
        const float* b = in[(i + 1) % n];
        const float da = below ? pos - a[axis] : a[axis] - pos;
        const float db = below ? pos - b[axis] : b[axis] - pos;
        if (da >= 0.f) {
            for (int k = 0; k < 3; ++k) out[m][k] = a[k];
            ++m;
        }
        if ((da >= 0.f) != (db >= 0.f)) {
            const float t = da / (da - db);
            for (int k = 0; k < 3; ++k) out[m][k] = a[k] + t * (b[k] - a[k]);
            out[m][axis] = pos;
            ++m;
        }
    }
    return m;
}

double tri_area(const Mesh& m, int64_t t) {
    const V3 a = m.vert(m.i[3 * t]), b = m.vert(m.i[3 * t + 1]), c = m.vert(m.i[3 * t + 2]);
    const V3 n = cross(b - a, c - a);
    return 0.5 * std::sqrt((double)n.x * n.x + (double)n.y * n.y + (double)n.z * n.z);
}

void split_into(const float (*poly)[3], int n, const BBox& box, int frags, int32_t id, std::vector<PrimRef>& out) {
    if (frags <= 1 || n == 0) {
        if (n == 0) return;
        PrimRef p{};
        for (int a = 0; a < 3; ++a) { p.lo[a] = INFINITY; p.hi[a] = -INFINITY; }
        for (int i = 0; i < n; ++i)
            for (int a = 0; a < 3; ++a) { p.lo[a] = fmn(p.lo[a], poly[i][a]); p.hi[a] = fmx(p.hi[a], poly[i][a]); }
        for (int a = 0; a < 3; ++a) {  // stay inside the parent box (clipping rounds)
            p.lo[a] = fmx(p.lo[a], box.lo[a]);
            p.hi[a] = fmn(p.hi[a], box.hi[a]);
            if (p.lo[a] > p.hi[a]) p.lo[a] = p.hi[a];
        }
        p.id = id;
        out.push_back(p);
        return;
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
        if (box.hi[a] - box.lo[a] > box.hi[axis] - box.lo[axis]) axis = a;
    const float mid = 0.5f * (box.lo[axis] + box.hi[axis]);
    float lp[12][3], rp[12][3];
    const int nl = clip_polygon(poly, n, axis, mid, true, lp);
    const int nr = clip_polygon(poly, n, axis, mid, false, rp);
    BBox lb = box, rb = box;
    lb.hi[axis] = mid;
    rb.lo[axis] = mid;
    split_into(lp, nl, lb, frags / 2, id, out);
    split_into(rp, nr, rb, frags / 2, id, out);
}

std::vector<PrimRef> make_refs(const Mesh& m, int max_frags) {
    const int64_t nt = m.nt();
    std::vector<PrimRef> refs(nt);
    std::vector<std::pair<float, int32_t>> fit;  // (box area / triangle area, triangle)
    for (int64_t t = 0; t < nt; ++t) {
        PrimRef& p = refs[t];
        for (int a = 0; a < 3; ++a) { p.lo[a] = INFINITY; p.hi[a] = -INFINITY; }
        for (int k = 0; k < 3; ++k) {
            const float* v = &m.v[3 * (size_t)m.i[3 * t + k]];
            for (int a = 0; a < 3; ++a) { p.lo[a] = fmn(p.lo[a], v[a]); p.hi[a] = fmx(p.hi[a], v[a]); }
        }
        p.id = (int32_t)t;
        p.pad = 0;
        if (max_frags > 1) {
            BBox b;
            b.grow(p.lo, p.hi);
            const double at = tri_area(m, t);
            if (at > 0.0) fit.push_back({(float)(b.area() / (2.0 * at)), (int32_t)t});
        }
    }
    if (max_frags <= 1 || fit.empty()) return refs;
    // Worst fit first; a box at most 4x the triangle's area is left alone.
    std::sort(fit.begin(), fit.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
    int64_t budget = nt;
    std::vector<PrimRef> extra;
    std::vector<uint8_t> replaced(nt, 0);
    for (const auto& [ratio, t] : fit) {
        if (ratio <= 4.0f || budget <= 0) break;
        float poly[3][3];
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) poly[k][a] = m.v[3 * (size_t)m.i[3 * (int64_t)t + k] + a];
        BBox b;
        b.grow(refs[t].lo, refs[t].hi);
        const size_t before = extra.size();
        split_into(poly, 3, b, max_frags, t, extra);
        const int64_t added = (int64_t)(extra.size() - before);
        if (added <= 1) {
            extra.resize(before);
            continue;
        }
        replaced[t] = 1;
        budget -= added - 1;
    }
    std::vector<PrimRef> out;
    out.reserve(nt + extra.size());
    for (int64_t t = 0; t < nt; ++t)
        if (!replaced[t]) out.push_back(refs[t]);
    out.insert(out.end(), extra.begin(), extra.end());
    return out;
}

}  // namespace

static void build_from_refs(std::vector<PrimRef> refs, const Mesh* mesh, float split_budget, int max_leaf, int bins,
                            int max_depth, bool big_leaves, int threads, Tree<2>& out) {
    Builder2 b;
    b.mesh = split_budget > 0.f ? mesh : nullptr;
    b.max_leaf = max_leaf;
    b.big_leaves = big_leaves;
    b.bins = std::max(2, std::min(bins, kMaxBins));
    b.max_depth = max_depth;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    b.spare_threads = threads - 1;
    b.threads_total = threads;
    b.refs = std::move(refs);
    const int64_t nt = (int64_t)b.refs.size();
    BBox all, call;
    for (const PrimRef& p : b.refs) {
        float c[3];
        centroid(p, c);
        all.grow(p.lo, p.hi);
        call.grow_pt(c);
    }
    // Spatial splits may add up to split_budget * nt duplicate references.
    const int64_t cap = b.mesh ? nt + (int64_t)((double)split_budget * (double)nt) : nt;
    b.refs.resize((size_t)cap);
    b.root_area = all.area();
    b.nodes.resize(std::max<int64_t>(1, cap));
    b.leaves.resize(std::max<int64_t>(1, cap));

    out = Tree<2>();
    out.bounds.lo = v3(all.lo[0], all.lo[1], all.lo[2]);
    out.bounds.hi = v3(all.hi[0], all.hi[1], all.hi[2]);
    if (nt == 0) {
        out.root_is_leaf = true;
        out.leaves.push_back(Leaf{0, 0});
        return;
    }
    const int32_t root = b.build(0, nt, cap, all, call, 0);
    // Slots are handed out in parallel; the root took slot 0.
    b.nodes.resize(b.n_nodes.load());
    b.leaves.resize(b.n_leaves.load());
    // Leaves index refs with slack between subtrees: pack their references.
    out.prim_refs.reserve((size_t)nt);
    for (Leaf& l : b.leaves) {
        const int32_t first = (int32_t)out.prim_refs.size();
        for (int32_t k = 0; k < l.count; ++k) out.prim_refs.push_back(b.refs[(size_t)l.first + k].id);
        l.first = first;
    }
    if (root < 0) {
        out.root_is_leaf = true;
        out.leaves.push_back(b.leaves[-root - 2]);
        return;
    }
    out.nodes = std::move(b.nodes);
    out.leaves = std::move(b.leaves);
}

void build_bvh2_tree(const Mesh& m, int max_leaf, int bins, int max_depth, bool big_leaves, int threads,
                     Tree<2>& out, int max_frags, float split_budget) {
    build_from_refs(make_refs(m, max_frags), &m, split_budget, max_leaf, bins, max_depth, big_leaves, threads, out);
}

void build_bvh2_tree_boxes(const float* boxes, int64_t n, int bins, int max_depth, int threads, Tree<2>& out) {
    std::vector<PrimRef> refs((size_t)n);
    for (int64_t k = 0; k < n; ++k) {
        PrimRef& p = refs[(size_t)k];
        for (int a = 0; a < 3; ++a) {
            p.lo[a] = boxes[6 * k + a];
            p.hi[a] = boxes[6 * k + 3 + a];
        }
        p.id = (int32_t)k;
        p.pad = 0;
    }
    build_from_refs(std::move(refs), nullptr, 0.f, 1, bins, max_depth, false, threads, out);
}

// ------------------------------------------------- treelet restructuring --
// Karras and Aila, "Fast Parallel Construction of High-Quality Bounding
// Volume Hierarchies" (HPG 2013), on the host's binary tree: at every inner
// node, bottom-up, a treelet of up to 7 leaves is grown by repeatedly opening
// its largest-area inner leaf; the binary topology over those leaves with the
// least SAH cost is found by dynamic programming over the 127 leaf subsets,
// and the treelet's inner nodes are rewired to it when that is cheaper.  The
// top-down binned build judges each split only by the bounds it sees at that
// level; rewiring fixes splits that later levels show to be poor (on terrain
// with thin overlapping boxes, far fewer nodes are entered per ray).  Leaves
// and their triangles are untouched, so every answer is the same.
namespace {
constexpr int kTreeletLeaves = 7;

struct TreeletOpt {
    Tree<2>& t;
    std::vector<float> cost;      // SAH cost of each inner node's subtree
    std::vector<uint8_t> dirty;   // the subtree changed in the latest pass that visited it

    explicit TreeletOpt(Tree<2>& tree) : t(tree), cost(tree.nodes.size(), 0.f), dirty(tree.nodes.size(), 1) {}

    static float area(const BBox& b) { return b.area(); }
    static BBox child_box(const TreeNode<2>& nd, int c) {
        BBox b;
        b.grow(nd.lo[c], nd.hi[c]);
        return b;
    }
    float code_cost(int32_t code, float a) const {
        return code >= 0 ? cost[(size_t)code] : kIntersectCost * a * (float)t.leaves[-code - 2].count;
    }
    void update_cost(int32_t v) {
        const TreeNode<2>& nd = t.nodes[v];
        const BBox b0 = child_box(nd, 0), b1 = child_box(nd, 1);
        BBox b = b0;
        b.grow(b1);
        cost[(size_t)v] = kTraversalCost * b.area() + code_cost(nd.child[0], b0.area()) +
                          code_cost(nd.child[1], b1.area());
    }

    // Rewires the treelet rooted at v (v keeps its index and its box) and
    // marks its inner nodes dirty; false when the treelet is kept.
    bool restructure(int32_t v) {
        int32_t code[kTreeletLeaves];
        BBox box[kTreeletLeaves];
        int32_t inner[kTreeletLeaves - 1];
        int nl = 2, ni = 1;
        inner[0] = v;
        for (int c = 0; c < 2; ++c) {
            code[c] = t.nodes[v].child[c];
            box[c] = child_box(t.nodes[v], c);
        }
        while (nl < kTreeletLeaves) {
            int pick = -1;
            float best_area = -1.f;
            for (int i = 0; i < nl; ++i)
                if (code[i] >= 0 && box[i].area() > best_area) { best_area = box[i].area(); pick = i; }
            if (pick < 0) break;
            const TreeNode<2>& nd = t.nodes[code[pick]];
            inner[ni++] = code[pick];
            code[nl] = nd.child[1];
            box[nl] = child_box(nd, 1);
            code[pick] = nd.child[0];
            box[pick] = child_box(nd, 0);
            ++nl;
        }
        if (nl < 3) return false;  // two leaves have one topology
        const unsigned full = (1u << nl) - 1u;
        BBox sbox[1 << kTreeletLeaves];
        float copt[1 << kTreeletLeaves];
        uint8_t part[1 << kTreeletLeaves];
        // A proper subset is numerically smaller than its set, so ascending
        // order has every part's cost ready.
        for (unsigned s = 1; s <= full; ++s) {
            const unsigned low = s & (0u - s);
            if (s == low) {
                const int i = __builtin_ctz(s);
                sbox[s] = box[i];
                copt[s] = code_cost(code[i], box[i].area());
                part[s] = 0;
                continue;
            }
            sbox[s] = sbox[s ^ low];
            sbox[s].grow(sbox[low]);
            float best = INFINITY;
            unsigned bp = 0;
            // each unordered split once: p holds the lowest leaf plus a proper
            // subset q of the others
            const unsigned rest = s ^ low;
            for (unsigned q = (rest - 1u) & rest;; q = (q - 1u) & rest) {
                const unsigned p = q | low;
                const float c = copt[p] + copt[s ^ p];
                if (c < best) { best = c; bp = p; }
                if (q == 0u) break;
            }
            copt[s] = kTraversalCost * sbox[s].area() + best;
            part[s] = (uint8_t)bp;
        }
        // Keep the current treelet unless the new one is clearly cheaper
        // (also when a cost is not finite).
        if (!(copt[full] < cost[(size_t)v] * (1.f - 1e-6f))) return false;
        int used = 0;
        emit(full, code, sbox, copt, part, inner, used);
        for (int k = 0; k < ni; ++k) dirty[(size_t)inner[k]] = 1;
        return true;
    }

    int32_t emit(unsigned s, const int32_t* code, const BBox* sbox, const float* copt, const uint8_t* part,
                 const int32_t* inner, int& used) {
        if ((s & (s - 1u)) == 0u) return code[__builtin_ctz(s)];
        const int32_t me = inner[used++];
        const unsigned p = part[s];
        const int32_t c0 = emit(p, code, sbox, copt, part, inner, used);
        const int32_t c1 = emit(s ^ p, code, sbox, copt, part, inner, used);
        TreeNode<2>& nd = t.nodes[me];
        nd.child[0] = c0;
        nd.child[1] = c1;
        for (int a = 0; a < 3; ++a) {
            nd.lo[0][a] = sbox[p].lo[a];
            nd.hi[0][a] = sbox[p].hi[a];
            nd.lo[1][a] = sbox[s ^ p].lo[a];
            nd.hi[1][a] = sbox[s ^ p].hi[a];
        }
        cost[(size_t)me] = copt[s];
        return me;
    }

    // Post-order of the dirty part of the subtree of `root` (a clean node's
    // subtree is clean).
    void post_order(int32_t root, std::vector<int32_t>& order) const {
        if (!dirty[(size_t)root]) return;
        std::vector<std::pair<int32_t, bool>> st{{root, false}};
        while (!st.empty()) {
            auto [v, done] = st.back();
            st.pop_back();
            if (done) {
                order.push_back(v);
                continue;
            }
            st.push_back({v, true});
            for (int c = 0; c < 2; ++c) {
                const int32_t ch = t.nodes[v].child[c];
                if (ch >= 0 && dirty[(size_t)ch]) st.push_back({ch, false});
            }
        }
    }

    // Costs bottom-up, then the treelet of every inner node with its subtree
    // already done.  A node whose subtree did not change in the previous pass
    // (and whose own treelet was kept) would keep it again, so only dirty
    // nodes are visited.  A restructure at v only rewires v's subtree, so
    // subtrees below a depth cut run on worker threads and the nodes above
    // them follow in reverse pre-order; the result is the same for any
    // thread count.
    void pass(int threads) {
        const size_t n = t.nodes.size();
        auto visit = [&](int32_t v) {
            if (!dirty[(size_t)v]) return;
            update_cost(v);
            if (restructure(v)) return;  // marked dirty by the rewiring
            const TreeNode<2>& nd = t.nodes[v];
            dirty[(size_t)v] = (uint8_t)((nd.child[0] >= 0 && dirty[(size_t)nd.child[0]]) ||
                                         (nd.child[1] >= 0 && dirty[(size_t)nd.child[1]]));
        };
        if (threads == 1 || n < 65536) {
            std::vector<int32_t> order;
            order.reserve(n);
            post_order(0, order);
            for (int32_t v : order) visit(v);
            return;
        }
        int depth_cut = 3;
        while ((1 << depth_cut) < 8 * threads) ++depth_cut;
        std::vector<int32_t> frontier, top;
        std::vector<std::pair<int32_t, int>> st{{0, 0}};
        while (!st.empty()) {
            const auto [v, d] = st.back();
            st.pop_back();
            if (d == depth_cut) {
                frontier.push_back(v);
                continue;
            }
            top.push_back(v);
            for (int c = 0; c < 2; ++c)
                if (t.nodes[v].child[c] >= 0) st.push_back({t.nodes[v].child[c], d + 1});
        }
        parallel_tasks((int64_t)frontier.size(), threads, [&](int64_t i) {
            std::vector<int32_t> sub;
            post_order(frontier[(size_t)i], sub);
            for (int32_t v : sub) visit(v);
        });
        for (auto it = top.rbegin(); it != top.rend(); ++it) visit(*it);
    }
};
}  // namespace

void treelet_optimize(Tree<2>& t, int passes, int threads) {
    if (passes <= 0 || t.root_is_leaf || t.nodes.empty()) return;
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    TreeletOpt opt(t);
    for (int p = 0; p < passes; ++p) opt.pass(threads);
}

// Optimal collapse of a binary tree into an 8-wide tree under a surface-area
// cost model.  For every binary node n and k = 1..8, best[n][k] is the least
// cost of representing the subtree of n with at most k children ("slots") of
// an 8-wide node:
//   k = 1:  one leaf holding all of n's triangles (when there are <= 3), or
//           an 8-wide node of its own: kNodeCost * area(n) plus n's two
//           children distributed over 8 slots;
//   k > 1:  the k = 1 choice, or n opened: best[c0][j] + best[c1][k - j].
// A leaf costs kLeafCost * area * triangles.  The choices are replayed
// top-down to emit the nodes.  Compared with greedily opening the largest
// child this fills the slots (fewer, fuller nodes) and merges small subtrees
// into leaves of up to 3 triangles.
namespace {
constexpr float kNodeCost = 1.0f;
constexpr float kLeafCost = 0.3f;

struct Collapse {
    struct Child {
        int32_t code;  // binary child code
        const float* lo;
        const float* hi;
    };

    const Tree<2>& t;
    std::vector<float> best;   // [node * 9 + k], k = 1..8
    std::vector<uint8_t> how;  // [node * 9 + k]: 0 leaf, 1 own node, 2 + j opened with j slots to child 0
    std::vector<uint8_t> node_split;  // slots to child 0 when the node is an 8-wide node of its own
    std::vector<int32_t> prims;

    explicit Collapse(const Tree<2>& tree) : t(tree) {}

    static float box_area(const float* lo, const float* hi) {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0.f && dy >= 0.f && dz >= 0.f)) return 0.f;
        return 2.f * (dx * dy + dy * dz + dz * dx);
    }
    int32_t count_of(int32_t code) const { return code >= 0 ? prims[code] : t.leaves[-code - 2].count; }
    float cost(int32_t code, int k, float a) const {
        if (code >= 0) return best[(size_t)code * 9 + k];
        return kLeafCost * a * (float)t.leaves[-code - 2].count;  // a binary leaf stays one leaf
    }

    // Post-order of the subtree of `root` (parallel builds interleave node numbering).
    void post_order(int32_t root, std::vector<int32_t>& order) const {
        std::vector<std::pair<int32_t, bool>> st{{root, false}};
        while (!st.empty()) {
            auto [v, done] = st.back();
            st.pop_back();
            if (done) {
                order.push_back(v);
                continue;
            }
            st.push_back({v, true});
            for (int c = 0; c < 2; ++c)
                if (t.nodes[v].child[c] >= 0) st.push_back({t.nodes[v].child[c], false});
        }
    }

    // The subtrees below depth D are solved on worker threads (about 8 per
    // thread for a balanced tree), then the nodes above them in post-order.
    void run(int threads) {
        const size_t n = t.nodes.size();
        best.assign(n * 9, INFINITY);
        how.assign(n * 9, 0);
        node_split.assign(n, 4);
        prims.assign(n, 0);
        if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
        if (threads == 1 || n < 65536) {
            std::vector<int32_t> order;
            order.reserve(n);
            post_order(0, order);
            for (int32_t v : order) solve(v);
            return;
        }
        int depth_cut = 3;
        while ((1 << depth_cut) < 8 * threads) ++depth_cut;
        std::vector<int32_t> frontier, top;  // top: nodes above the cut, in pre-order
        std::vector<std::pair<int32_t, int>> st{{0, 0}};
        while (!st.empty()) {
            const auto [v, d] = st.back();
            st.pop_back();
            if (d == depth_cut) {
                frontier.push_back(v);
                continue;
            }
            top.push_back(v);
            for (int c = 0; c < 2; ++c)
                if (t.nodes[v].child[c] >= 0) st.push_back({t.nodes[v].child[c], d + 1});
        }
        parallel_tasks((int64_t)frontier.size(), threads, [&](int64_t i) {
            std::vector<int32_t> sub;
            post_order(frontier[(size_t)i], sub);
            for (int32_t v : sub) solve(v);
        });
        // Reverse pre-order visits children before parents.
        for (auto it = top.rbegin(); it != top.rend(); ++it) solve(*it);
    }

    // best / how / prims of node v from its children's.
    void solve(int32_t v) {
        const TreeNode<2>& nd = t.nodes[v];
        const float ca[2] = {box_area(nd.lo[0], nd.hi[0]), box_area(nd.lo[1], nd.hi[1])};
        BBox b;
        b.grow(nd.lo[0], nd.hi[0]);
        b.grow(nd.lo[1], nd.hi[1]);
        const float av = b.area();
        prims[v] = count_of(nd.child[0]) + count_of(nd.child[1]);
        float open[9];
        uint8_t split[9];
        for (int k = 2; k <= 8; ++k) {
            open[k] = INFINITY;
            split[k] = 1;
            for (int j = 1; j < k; ++j) {
                const float c = cost(nd.child[0], j, ca[0]) + cost(nd.child[1], k - j, ca[1]);
                if (c < open[k]) { open[k] = c; split[k] = (uint8_t)j; }
            }
        }
        float* bv = &best[(size_t)v * 9];
        uint8_t* hv = &how[(size_t)v * 9];
        const float as_node = kNodeCost * av + open[8];
        node_split[v] = split[8];
        const float as_leaf = prims[v] <= 3 ? kLeafCost * av * (float)prims[v] : INFINITY;
        bv[1] = std::min(as_leaf, as_node);
        hv[1] = as_leaf <= as_node ? 0 : 1;
        for (int k = 2; k <= 8; ++k) {
            bv[k] = bv[k - 1];
            hv[k] = hv[k - 1];
            if (open[k] < bv[k]) { bv[k] = open[k]; hv[k] = (uint8_t)(2 + split[k]); }
        }
    }

    // Triangles of a binary subtree appended to refs, each once from `first` on
    // (fragments of one pre-split triangle can sit in sibling leaves).
    void gather(int32_t code, std::vector<int32_t>& refs, size_t first) const {
        if (code < 0) {
            const Leaf& l = t.leaves[-code - 2];
            for (int32_t k = 0; k < l.count; ++k) {
                const int32_t id = t.prim_refs[l.first + k];
                if (std::find(refs.begin() + first, refs.end(), id) == refs.end()) refs.push_back(id);
            }
            return;
        }
        gather(t.nodes[code].child[0], refs, first);
        gather(t.nodes[code].child[1], refs, first);
    }

    // The slots that the binary child `code` (box lo/hi) fills given k slots.
    void slots(int32_t code, int k, const float* lo, const float* hi, std::vector<Child>& out) const {
        if (code >= 0 && how[(size_t)code * 9 + k] >= 2) {
            const TreeNode<2>& nd = t.nodes[code];
            const int j = how[(size_t)code * 9 + k] - 2;
            slots(nd.child[0], j, nd.lo[0], nd.hi[0], out);
            slots(nd.child[1], k - j, nd.lo[1], nd.hi[1], out);
            return;
        }
        out.push_back(Child{code, lo, hi});
    }
};
}  // namespace

// Emits the 8-wide subtree of binary node `src` into `frag` (its node 0).
// With split_grain > 0, inner children of at most split_grain triangles are
// not expanded but listed in `pending` (fragment node, slot, binary node), to
// be emitted as fragments of their own.
struct Pending {
    int32_t node;
    int slot;
    int32_t src;
};

static void emit_subtree(const Collapse& cl, int32_t src, Tree<8>& frag, int64_t split_grain,
                         std::vector<Pending>* pending) {
    const Tree<2>& t2 = cl.t;
    std::vector<std::pair<int32_t, int32_t>> work{{src, 0}};  // (binary node, 8-wide node)
    frag.nodes.push_back(TreeNode<8>{});
    while (!work.empty()) {
        const auto [s, dst] = work.back();
        work.pop_back();
        const TreeNode<2>& nd = t2.nodes[s];
        const int j = cl.node_split[s];  // an 8-wide node opens its binary node into 8 slots
        std::vector<Collapse::Child> ch;
        cl.slots(nd.child[0], j, nd.lo[0], nd.hi[0], ch);
        cl.slots(nd.child[1], 8 - j, nd.lo[1], nd.hi[1], ch);
        TreeNode<8> d{};
        for (int k = 0; k < 8; ++k) d.child[k] = -1;
        d.count = (int)ch.size();
        for (size_t c = 0; c < ch.size(); ++c) {
            for (int a = 0; a < 3; ++a) { d.lo[c][a] = ch[c].lo[a]; d.hi[c][a] = ch[c].hi[a]; }
            const int32_t code = ch[c].code;
            if (code >= 0 && cl.how[(size_t)code * 9 + 1] == 1) {
                if (split_grain > 0 && cl.prims[code] <= split_grain) {
                    pending->push_back(Pending{dst, (int)c, code});
                    d.child[c] = 0;  // filled in when the fragments are joined
                    continue;
                }
                const int32_t ni = (int32_t)frag.nodes.size();
                frag.nodes.push_back(TreeNode<8>{});
                work.push_back({code, ni});
                d.child[c] = ni;
            } else {
                // A binary leaf, or a subtree merged into one leaf (<= 3 triangles).
                const int32_t first = (int32_t)frag.prim_refs.size();
                cl.gather(code, frag.prim_refs, (size_t)first);
                const int32_t leaf = (int32_t)frag.leaves.size();
                frag.leaves.push_back(Leaf{first, (int32_t)frag.prim_refs.size() - first});
                d.child[c] = -(leaf + 2);
            }
        }
        frag.nodes[dst] = d;
    }
}

// Appends fragment f to out (renumbering its nodes, leaves and references);
// returns the index its root got.
static int32_t join_fragment(Tree<8>& out, const Tree<8>& f) {
    const int32_t node_off = (int32_t)out.nodes.size(), leaf_off = (int32_t)out.leaves.size();
    const int32_t ref_off = (int32_t)out.prim_refs.size();
    for (TreeNode<8> nd : f.nodes) {
        for (int c = 0; c < 8; ++c) {
            if (nd.child[c] >= 0) nd.child[c] += node_off;
            else if (nd.child[c] <= -2) nd.child[c] -= leaf_off;
        }
        out.nodes.push_back(nd);
    }
    for (Leaf l : f.leaves) {
        l.first += ref_off;
        out.leaves.push_back(l);
    }
    out.prim_refs.insert(out.prim_refs.end(), f.prim_refs.begin(), f.prim_refs.end());
    return node_off;
}

// The 8-wide tree is the same for any thread count (node numbering aside):
// large trees are emitted as a top fragment plus one fragment per subtree of
// at most `grain` triangles, converted independently and joined.
static void collapse_optimal(const Tree<2>& t2, Tree<8>& out, int threads) {
    Collapse cl(t2);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    cl.run(threads);
    out = Tree<8>();
    out.bounds = t2.bounds;
    const int64_t total = cl.prims[0];
    const int64_t grain = std::max<int64_t>(16384, total / (8 * (int64_t)threads));
    if (threads == 1 || total <= 2 * grain) {
        emit_subtree(cl, 0, out, 0, nullptr);
        return;
    }
    std::vector<Pending> pending;
    emit_subtree(cl, 0, out, grain, &pending);
    std::vector<Tree<8>> frags(pending.size());
    parallel_tasks((int64_t)pending.size(), threads,
                   [&](int64_t i) { emit_subtree(cl, pending[(size_t)i].src, frags[(size_t)i], 0, nullptr); });
    for (size_t i = 0; i < pending.size(); ++i)
        out.nodes[pending[i].node].child[pending[i].slot] = join_fragment(out, frags[i]);
}

void collapse_to_bvh8(const Tree<2>& t2, Tree<8>& out, int threads) {
    out = Tree<8>();
    out.bounds = t2.bounds;
    out.prim_refs = t2.prim_refs;
    out.leaves = t2.leaves;
    if (t2.root_is_leaf) {
        // A single-leaf scene becomes an inner root with one leaf child.
        TreeNode<8> r{};
        for (int k = 0; k < 8; ++k) r.child[k] = -1;
        const bool empty = t2.leaves.empty() || t2.leaves[0].count == 0;
        r.count = empty ? 0 : 1;
        r.child[0] = empty ? -1 : -2;
        r.lo[0][0] = t2.bounds.lo.x; r.lo[0][1] = t2.bounds.lo.y; r.lo[0][2] = t2.bounds.lo.z;
        r.hi[0][0] = t2.bounds.hi.x; r.hi[0][1] = t2.bounds.hi.y; r.hi[0][2] = t2.bounds.hi.z;
        out.nodes.push_back(r);
        return;
    }
    collapse_optimal(t2, out, threads);
}

template <int W>
static int depth_of(const Tree<W>& t) {
    if (t.root_is_leaf || t.nodes.empty()) return 1;
    std::vector<std::pair<int32_t, int>> st{{0, 1}};
    int best = 1;
    while (!st.empty()) {
        auto [n, d] = st.back();
        st.pop_back();
        const auto& nd = t.nodes[n];
        for (int c = 0; c < W; ++c) {
            if (nd.child[c] >= 0) st.push_back({nd.child[c], d + 1});
            else if (nd.child[c] <= -2) best = std::max(best, d + 1);
        }
    }
    return best;
}

int tree_depth2(const Tree<2>& t) { return depth_of(t); }
int tree_depth8(const Tree<8>& t) { return depth_of(t); }

}  // namespace rq
