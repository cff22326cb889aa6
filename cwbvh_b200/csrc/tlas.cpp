// Host side of two-level scenes: the top-level CWBVH over instances.
//
// Each instance's world bounds are the 8 corners of its bottom-level scene's
// bounds put through the object-to-world transform in double precision and
// rounded outwards to float, so the top-level boxes contain the instance's
// geometry; the binned SAH builder and the cost-driven 8-wide collapse run
// on those boxes, and the converter emits, in place of each leaf triangle's
// Woop rows, the instance's world-to-object rows (the affine inverse,
// computed in double and rounded once).
#include <algorithm>
#include <cmath>
#include <limits>
#include <memory>
#include <new>
#include <vector>

#include "host_common.h"

using namespace rq;

namespace {

// Inverse of a 3x4 row-major affine transform in double; false if it is
// singular (|det| below 1e-12 of the scale of its linear part cubed).
bool invert_affine(const float* m, double inv[12]) {
    const double a = m[0], b = m[1], c = m[2], d = m[4], e = m[5], f = m[6], g = m[8], h = m[9], k = m[10];
    const double c00 = e * k - f * h, c01 = f * g - d * k, c02 = d * h - e * g;
    const double det = a * c00 + b * c01 + c * c02;
    const double scale = std::max({std::fabs(a), std::fabs(b), std::fabs(c), std::fabs(d), std::fabs(e),
                                   std::fabs(f), std::fabs(g), std::fabs(h), std::fabs(k)});
    if (!std::isfinite(det) || !(std::fabs(det) > 1e-12 * scale * scale * scale)) return false;
    const double r = 1.0 / det;
    const double l[9] = {c00 * r, (c * h - b * k) * r, (b * f - c * e) * r,
                         c01 * r, (a * k - c * g) * r, (c * d - a * f) * r,
                         c02 * r, (b * g - a * h) * r, (a * e - b * d) * r};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) inv[4 * i + j] = l[3 * i + j];
        inv[4 * i + 3] = -(l[3 * i] * m[3] + l[3 * i + 1] * m[7] + l[3 * i + 2] * m[11]);
    }
    return true;
}

}  // namespace

extern "C" rq_status rq_tlas_build_host(const float* blas_bounds, int n_blas, const float* object_to_world,
                                        const int32_t* blas_index, int64_t n_instances, rq_host_bvh_t* out) {
    if (!out || !blas_bounds || n_blas <= 0 || n_instances <= 0 || !object_to_world || !blas_index ||
        n_instances > (int64_t)std::numeric_limits<int32_t>::max() / 3)
        return RQ_ERR_INVALID_ARG;
    for (int64_t j = 0; j < 6 * (int64_t)n_blas; ++j)
        if (!std::isfinite(blas_bounds[j])) return RQ_ERR_INVALID_ARG;
    try {
        std::vector<float> rows((size_t)n_instances * 12), boxes((size_t)n_instances * 6);
        for (int64_t k = 0; k < n_instances; ++k) {
            const int32_t b = blas_index[k];
            if (b < 0 || b >= n_blas) return RQ_ERR_INVALID_ARG;
            const float* m = object_to_world + 12 * k;
            for (int j = 0; j < 12; ++j)
                if (!std::isfinite(m[j])) return RQ_ERR_INVALID_ARG;
            double inv[12];
            if (!invert_affine(m, inv)) return RQ_ERR_INVALID_ARG;
            for (int j = 0; j < 12; ++j) rows[12 * k + j] = (float)inv[j];
            const float* bb = blas_bounds + 6 * (int64_t)b;
            double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
            for (int c = 0; c < 8; ++c) {
                const double p[3] = {(c & 1) ? bb[3] : bb[0], (c & 2) ? bb[4] : bb[1], (c & 4) ? bb[5] : bb[2]};
                for (int i = 0; i < 3; ++i) {
                    const double w = (double)m[4 * i] * p[0] + (double)m[4 * i + 1] * p[1] +
                                     (double)m[4 * i + 2] * p[2] + (double)m[4 * i + 3];
                    lo[i] = std::min(lo[i], w);
                    hi[i] = std::max(hi[i], w);
                }
            }
            for (int i = 0; i < 3; ++i) {
                boxes[6 * k + i] = std::nextafter((float)lo[i], -INFINITY);
                boxes[6 * k + 3 + i] = std::nextafter((float)hi[i], INFINITY);
            }
        }
        std::unique_ptr<rq_host_bvh> r(new rq_host_bvh());
        Tree<2> t2;
        build_bvh2_tree_boxes(boxes.data(), n_instances, 32, 64, 0, t2);
        collapse_to_bvh8(t2, r->b.tree8);
        convert_cwbvh_instances(r->b.tree8, rows.data(), blas_index, r->b);
        r->b.depth = tree_depth8(r->b.tree8);
        r->b.has_tree = true;
        *out = r.release();
        return RQ_OK;
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}
