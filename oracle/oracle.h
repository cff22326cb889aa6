/*
 * oracle.h -- CPU restatement of the reference's ray-query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This code is the checker: the parity tests, the
 * smoke check and the CPU-baseline leg of bench.py call it; the product
 * library (librq.so) never links, loads or calls it.
 *
 * Buffers use the reference layouts (src/helper_math.h:1853-1865,
 * src/GPUBVHConverter.cpp:10-403): rays are 8 floats, hits 4 floats, nodes
 * and Woop rows float4.
 */
#ifndef RQ_ORACLE_H
#define RQ_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_CWBVH = 0, ORACLE_BVH2 = 1 };
enum { ORACLE_ERR_STACK = 1, ORACLE_ERR_BAD_SCENE = 4 };

/* Trace n rays; returns the OR of the per-ray error bits.  node_visits /
 * tri_tests may be NULL.  threads <= 0 uses all OpenMP threads. */
int oracle_trace(int kind, const float* nodes, int64_t node_f4, const float* woop, int64_t woop_f4,
                 const float* rays, int64_t n, int any_hit, float* hits, int32_t* node_visits,
                 int32_t* tri_tests, int threads);

/* Double-precision intersection of a ray with the triangle (v0, v1, v2) in
 * the Woop frame (point = v2 + u (v0 - v2) + v (v1 - v2)): out = t, u, v,
 * determinant.  Used to adjudicate disagreements. */
void oracle_tri_f64(const float ray[8], const float v0[3], const float v1[3], const float v2[3],
                    double out[4]);

/* AO rays from surfels, the same formulas and Philox4x32-10 stream as the
 * product's generator, with the host's sinf/cosf/sqrtf. */
void oracle_aorays(const float* pos, const float* nrm, const float* radius, int64_t n_surfels,
                   int spp, uint64_t seed, float tmin, float tmax, float offset_scale, float* out);

/* Philox4x32-10 block for counter (c0, c1, c2, c3) and key (k0, k1). */
void oracle_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]);

int oracle_max_threads(void);

#ifdef __cplusplus
}
#endif

#endif
