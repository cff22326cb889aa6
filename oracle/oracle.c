/*
 * oracle.c -- CPU restatement of the reference's traversal, Woop test and AO
 * ray generation.  TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for
 * the CUDA kernels, never part of the product.
 *
 * Arithmetic.  Every step follows the reference kernels' expressions in the
 * same order, with the products that a*b+c contracts into a fused
 * multiply-add written as fmaf() and everything else as single IEEE float
 * operations (built with -ffp-contract=off).  1/x is IEEE division; the
 * reference, built with -use_fast_math, uses an approximate reciprocal, so
 * against the reference itself t agrees to about an ulp (and ties are
 * adjudicated in double precision by oracle_tri_f64).
 *
 * Traversal order.  Per ray, no warp effects: the CWBVH loop is the
 * reference's with triangle postponing off, the BVH2 loop is the
 * reference's while-while with a one-lane vote (a ray stops its node loop as
 * soon as it holds a leaf).  Closest-hit results differ from a warp-ordered
 * traversal only on exact ties; any-hit occlusion does not depend on order.
 */
#include "oracle.h"

#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float x, y, z, w; } f4;

static inline uint32_t ubits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline int32_t ibits(float f) { int32_t i; memcpy(&i, &f, 4); return i; }
static inline float from_u(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline float from_i(int32_t i) { float f; memcpy(&f, &i, 4); return f; }

static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }
static inline int32_t imin(int32_t a, int32_t b) { return a < b ? a : b; }

/* Video-instruction min/max on float bits compared as signed ints
 * (src/FastDeviceMinMax.h:44-51). */
static inline float imax3f(float a, float b, float c) { return from_i(imax(imax(ibits(a), ibits(b)), ibits(c))); }
static inline float imin3f(float a, float b, float c) { return from_i(imin(imin(ibits(a), ibits(b)), ibits(c))); }
static inline float imin_max(float a, float b, float c) { return from_i(imax(imin(ibits(a), ibits(b)), ibits(c))); }
static inline float imax_min(float a, float b, float c) { return from_i(imin(imax(ibits(a), ibits(b)), ibits(c))); }

static inline unsigned bfind(uint32_t x) { return 31u - (unsigned)__builtin_clz(x); }

/* src/TraversalKernelCWBVH.cu:31,78-80 */
static inline float guarded_rcp(float d) {
    const float ooeps = 0x1p-80f;
    return 1.0f / (fabsf(d) > ooeps ? d : copysignf(ooeps, d));
}

/* src/TraversalKernelCWBVH.cu:322-347 (same acceptance test as
 * src/TraversalKernelBVH2.cu:135-158). */
static inline int woop_test(const f4* v, const float o[3], const float d[3], float tmin, float tmax, float* t,
                            float* u, float* vv) {
    const f4 a = v[0], b = v[1], c = v[2];
    const float Oz = fmaf(-o[2], a.z, fmaf(-o[1], a.y, fmaf(-o[0], a.x, a.w)));
    const float Dz = fmaf(d[2], a.z, fmaf(d[0], a.x, d[1] * a.y));
    const float tt = Oz * (1.0f / Dz);
    const float Ox = fmaf(o[2], b.z, fmaf(o[1], b.y, fmaf(o[0], b.x, b.w)));
    const float Dx = fmaf(d[2], b.z, fmaf(d[0], b.x, d[1] * b.y));
    const float uu = fmaf(tt, Dx, Ox);
    const float Oy = fmaf(o[2], c.z, fmaf(o[1], c.y, fmaf(o[0], c.x, c.w)));
    const float Dy = fmaf(d[2], c.z, fmaf(d[0], c.x, d[1] * c.y));
    const float v2 = fmaf(tt, Dy, Oy);
    *t = tt;
    *u = uu;
    *vv = v2;
    return (tt > tmin && tt < tmax) && (uu >= 0.0f && uu <= 1.0f) && (v2 >= 0.0f && uu + v2 <= 1.0f);
}

#define STACK_CAP 256

/* Node test of one CWBVH node (src/TraversalKernelCWBVH.cu:117-289): the next
 * node group (child base, inner hit bits | imask) and triangle group. */
static void cwbvh_visit(const f4* n, const float o[3], const float idir[3], uint32_t octinv, float tmin, float tmax,
                        uint32_t* ngx_, uint32_t* ngy_, uint32_t* tgx_, uint32_t* tgy_) {
    const uint32_t ew = ubits(n[0].w);
    float adj[3], org[3];
    for (int a = 0; a < 3; ++a) {
        const int e = (int)(int8_t)((ew >> (8 * a)) & 0xFFu);
        adj[a] = from_u(((uint32_t)(e + 127)) << 23) * idir[a];
    }
    org[0] = -(o[0] - n[0].x) * idir[0];
    org[1] = -(o[1] - n[0].y) * idir[1];
    org[2] = -(o[2] - n[0].z) * idir[2];
    uint32_t hitmask = 0;
    for (int c = 0; c < 8; ++c) {
        const int g = c >> 2, k = c & 3;
        const uint32_t meta = (ubits(g ? n[1].w : n[1].z) >> (8 * k)) & 0xFFu;
        const int inner = (meta & 0x18u) == 0x18u;
        const uint32_t bitidx = (inner ? (meta ^ octinv) : meta) & 0x1Fu;
        const uint32_t cbits = (meta >> 5) & 7u;
        /* qlo/qhi words: x lo n2.x|n2.y, x hi n3.z|n3.w, y lo n2.z|n2.w,
         * y hi n4.x|n4.y, z lo n3.x|n3.y, z hi n4.z|n4.w */
        const uint32_t wl[3] = {ubits(g ? n[2].y : n[2].x), ubits(g ? n[2].w : n[2].z), ubits(g ? n[3].y : n[3].x)};
        const uint32_t wh[3] = {ubits(g ? n[3].w : n[3].z), ubits(g ? n[4].y : n[4].x), ubits(g ? n[4].w : n[4].z)};
        float t0[3], t1[3];
        for (int a = 0; a < 3; ++a) {
            const uint32_t lo = idir[a] < 0.f ? wh[a] : wl[a];
            const uint32_t hi = idir[a] < 0.f ? wl[a] : wh[a];
            t0[a] = fmaf((float)((lo >> (8 * k)) & 0xFFu), adj[a], org[a]);
            t1[a] = fmaf((float)((hi >> (8 * k)) & 0xFFu), adj[a], org[a]);
        }
        const float cmin = fmaxf(imax3f(t0[0], t0[1], t0[2]), tmin);
        const float cmax = fminf(imin3f(t1[0], t1[1], t1[2]), tmax);
        if (cmin <= cmax) hitmask |= cbits << bitidx;
    }
    *ngx_ = ubits(n[1].x);
    *ngy_ = (hitmask & 0xFF000000u) | (ew >> 24);
    *tgx_ = ubits(n[1].y);
    *tgy_ = hitmask & 0x00FFFFFFu;
}

/* One ray through the CWBVH (src/TraversalKernelCWBVH.cu:74-363). */
static int cwbvh_ray(const f4* nodes, int64_t node_f4, const f4* woop, int64_t woop_f4, const float* ray, int any,
                     float* hit, int32_t* nvis, int32_t* ntri) {
    const float o[3] = {ray[0], ray[1], ray[2]}, d[3] = {ray[4], ray[5], ray[6]};
    const float tmin = ray[3];
    float tmax = ray[7];
    const float idir[3] = {guarded_rcp(d[0]), guarded_rcp(d[1]), guarded_rcp(d[2])};
    const uint32_t octinv = 7u - (((d[0] < 0.f) ? 4u : 0u) | ((d[1] < 0.f) ? 2u : 0u) | ((d[2] < 0.f) ? 1u : 0u));
    uint32_t ngx = 0, ngy = 0x80000000u, tgx = 0, tgy = 0;
    uint32_t stx[STACK_CAP], sty[STACK_CAP];
    int sp = 0, hit_addr = -1, err = 0;
    float hu = 0.f, hv = 0.f;
    int32_t visits = 0, tests = 0;

    for (;;) {
        if (ngy > 0x00FFFFFFu) {
            const uint32_t hits = ngy;
            const unsigned bit = bfind(hits);
            const uint32_t base = ngx;
            ngy &= ~(1u << bit);
            if (ngy > 0x00FFFFFFu) {
                if (sp >= STACK_CAP) { err |= ORACLE_ERR_STACK; break; }
                stx[sp] = ngx; sty[sp] = ngy; ++sp;
            }
            const unsigned slot = (bit - 24u) ^ octinv;
            const uint32_t ci = base + (uint32_t)__builtin_popcount(hits & ~(0xFFFFFFFFu << slot));
            if ((uint64_t)ci * 5u + 5u > (uint64_t)node_f4) { err |= ORACLE_ERR_BAD_SCENE; break; }
            const f4* n = nodes + (size_t)ci * 5u;
            ++visits;
            cwbvh_visit(n, o, idir, octinv, tmin, tmax, &ngx, &ngy, &tgx, &tgy);
        } else {
            tgx = ngx; tgy = ngy;
            ngx = 0; ngy = 0;
        }
        int done = 0;
        while (tgy != 0) {
            const unsigned ti = bfind(tgy);
            const uint32_t tri = tgx * 3u + ti * 3u;
            tgy &= ~(1u << ti);
            if ((uint64_t)tri + 3u > (uint64_t)woop_f4) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
            ++tests;
            float t, u, v;
            if (woop_test(woop + tri, o, d, tmin, tmax, &t, &u, &v)) {
                tmax = t; hit_addr = (int)tri; hu = u; hv = v;
                if (any) { done = 1; break; }
            }
        }
        if (done) break;
        if (ngy <= 0x00FFFFFFu) {
            if (sp > 0) { --sp; ngx = stx[sp]; ngy = sty[sp]; }
            else break;
        }
    }
    if (err) hit_addr = -1;
    hit[0] = tmax; hit[1] = from_i(hit_addr); hit[2] = hu; hit[3] = hv;
    if (nvis) *nvis = visits;
    if (ntri) *ntri = tests;
    return err;
}

/* One ray through the BVH2 (src/TraversalKernelBVH2.cu:47-177). */
static int bvh2_ray(const f4* nodes, int64_t node_f4, const f4* woop, int64_t woop_f4, const float* ray, int any,
                    float* hit, int32_t* nvis, int32_t* ntri) {
    const int32_t SENT = 0x76543210;
    const float o[3] = {ray[0], ray[1], ray[2]}, d[3] = {ray[4], ray[5], ray[6]};
    const float tmin = ray[3];
    float tmax = ray[7];
    const float idir[3] = {guarded_rcp(d[0]), guarded_rcp(d[1]), guarded_rcp(d[2])};
    const float ood[3] = {o[0] * idir[0], o[1] * idir[1], o[2] * idir[2]};
    int32_t stack[STACK_CAP];
    int sp = 0;
    stack[0] = SENT;
    int32_t node = 0, leaf = 0;
    int hit_addr = -1, err = 0, done = 0;
    float hu = 0.f, hv = 0.f;
    int32_t visits = 0, tests = 0;
#define POP() (sp > 0 ? stack[sp--] : stack[0])
    while (node != SENT && !done) {
        leaf = 0;
        while (node != SENT && node >= 0 && leaf >= 0) {
            if ((uint64_t)(uint32_t)node + 4u > (uint64_t)node_f4) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
            const f4* n = nodes + node;
            ++visits;
            /* lo * idir - ood (src/TraversalKernelBVH2.cu:14-24) */
            const float a0[6] = {fmaf(n[0].x, idir[0], -ood[0]), fmaf(n[0].y, idir[0], -ood[0]),
                                 fmaf(n[0].z, idir[1], -ood[1]), fmaf(n[0].w, idir[1], -ood[1]),
                                 fmaf(n[2].x, idir[2], -ood[2]), fmaf(n[2].y, idir[2], -ood[2])};
            const float a1[6] = {fmaf(n[1].x, idir[0], -ood[0]), fmaf(n[1].y, idir[0], -ood[0]),
                                 fmaf(n[1].z, idir[1], -ood[1]), fmaf(n[1].w, idir[1], -ood[1]),
                                 fmaf(n[2].z, idir[2], -ood[2]), fmaf(n[2].w, idir[2], -ood[2])};
            const float c0min = imin_max(a0[4], a0[5], imin_max(a0[2], a0[3], imin_max(a0[0], a0[1], tmin)));
            const float c0max = imax_min(a0[4], a0[5], imax_min(a0[2], a0[3], imax_min(a0[0], a0[1], tmax)));
            const float c1min = imin_max(a1[4], a1[5], imin_max(a1[2], a1[3], imin_max(a1[0], a1[1], tmin)));
            const float c1max = imax_min(a1[4], a1[5], imax_min(a1[2], a1[3], imax_min(a1[0], a1[1], tmax)));
            const int t0 = c0min <= c0max, t1 = c1min <= c1max;
            int32_t cx = ibits(n[3].x), cy = ibits(n[3].y);
            if (!t0 && !t1) {
                node = POP();
            } else {
                node = t0 ? cx : cy;
                if (t0 && t1) {
                    if (c1min < c0min) { const int32_t tmp = node; node = cy; cy = tmp; }
                    if (sp + 1 >= STACK_CAP) { err |= ORACLE_ERR_STACK; done = 1; break; }
                    stack[++sp] = cy;
                }
            }
            if (node < 0 && leaf >= 0) {
                leaf = node;
                node = POP();
            }
        }
        while (!done && leaf < 0) {
            for (int32_t tri = ~leaf;; tri += 3) {
                if ((uint64_t)(uint32_t)tri + 1u > (uint64_t)woop_f4) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
                if (ubits(woop[tri].x) == 0x80000000u) break;
                if ((uint64_t)(uint32_t)tri + 3u > (uint64_t)woop_f4) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
                ++tests;
                float t, u, v;
                if (woop_test(woop + tri, o, d, tmin, tmax, &t, &u, &v)) {
                    tmax = t; hit_addr = tri; hu = u; hv = v;
                    if (any) { done = 1; break; }
                }
            }
            if (done) break;
            leaf = node;
            if (node < 0) node = POP();
        }
    }
#undef POP
    if (err) hit_addr = -1;
    hit[0] = tmax; hit[1] = from_i(hit_addr); hit[2] = hu; hit[3] = hv;
    if (nvis) *nvis = visits;
    if (ntri) *ntri = tests;
    return err;
}

int oracle_trace(int kind, const float* nodes, int64_t node_f4, const float* woop, int64_t woop_f4, const float* rays,
                 int64_t n, int any_hit, float* hits, int32_t* node_visits, int32_t* tri_tests, int threads) {
    int err = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) reduction(| : err) num_threads(threads)
#endif
    for (int64_t i = 0; i < n; ++i) {
        int32_t* nv = node_visits ? node_visits + i : NULL;
        int32_t* nt = tri_tests ? tri_tests + i : NULL;
        if (kind == ORACLE_CWBVH)
            err |= cwbvh_ray((const f4*)nodes, node_f4, (const f4*)woop, woop_f4, rays + 8 * i, any_hit, hits + 4 * i, nv, nt);
        else
            err |= bvh2_ray((const f4*)nodes, node_f4, (const f4*)woop, woop_f4, rays + 8 * i, any_hit, hits + 4 * i, nv, nt);
    }
    (void)threads;
    return err;
}

/* One ray through a two-level scene: a top-level CWBVH whose leaf "triangles"
 * are instances (3 rows of the world-to-object transform where the Woop rows
 * would be; map entries (instance, bottom-level index, -1)) over bottom-level
 * CWBVHs.  This is the library's own extension (the reference has no
 * instancing); the traversal order -- push the top level's node group, then
 * its instance group, enter the instance, leave it when its stack part is
 * empty -- is the one the GPU kernel follows. */
static int inst_ray(const f4* tn, int64_t tn_f4, const f4* rows, int64_t rows_f4, const int32_t* map, int n_blas,
                    const float* const* bn, const int64_t* bn_f4, const float* const* bw, const int64_t* bw_f4,
                    const float* ray, int any, float* hit, int32_t* inst_out) {
    const float wo[3] = {ray[0], ray[1], ray[2]}, wd[3] = {ray[4], ray[5], ray[6]};
    const float tmin = ray[3];
    float tmax = ray[7];
    float o[3], d[3], idir[3];
    uint32_t octinv;
    const f4* nodes = tn;
    const f4* woop = rows;
    int64_t node_f4 = tn_f4, woop_f4 = rows_f4;
    int in_blas = 0, inst_sp = 0, cur_inst = -1, hit_inst = -1;
#define SET_RAY(O, D)                                                                                         \
    do {                                                                                                      \
        for (int a_ = 0; a_ < 3; ++a_) { o[a_] = (O)[a_]; d[a_] = (D)[a_]; idir[a_] = guarded_rcp(d[a_]); } \
        octinv = 7u - (((d[0] < 0.f) ? 4u : 0u) | ((d[1] < 0.f) ? 2u : 0u) | ((d[2] < 0.f) ? 1u : 0u));     \
    } while (0)
    SET_RAY(wo, wd);
    uint32_t ngx = 0, ngy = 0x80000000u, tgx = 0, tgy = 0;
    uint32_t stx[STACK_CAP], sty[STACK_CAP];
    int sp = 0, hit_addr = -1, err = 0;
    float hu = 0.f, hv = 0.f;

    for (;;) {
        if (ngy > 0x00FFFFFFu) {
            const uint32_t hits = ngy;
            const unsigned bit = bfind(hits);
            const uint32_t base = ngx;
            ngy &= ~(1u << bit);
            if (ngy > 0x00FFFFFFu) {
                if (sp >= STACK_CAP) { err |= ORACLE_ERR_STACK; break; }
                stx[sp] = ngx; sty[sp] = ngy; ++sp;
            }
            const unsigned slot = (bit - 24u) ^ octinv;
            const uint32_t ci = base + (uint32_t)__builtin_popcount(hits & ~(0xFFFFFFFFu << slot));
            if ((uint64_t)ci * 5u + 5u > (uint64_t)node_f4) { err |= ORACLE_ERR_BAD_SCENE; break; }
            cwbvh_visit(nodes + (size_t)ci * 5u, o, idir, octinv, tmin, tmax, &ngx, &ngy, &tgx, &tgy);
        } else {
            tgx = ngx; tgy = ngy;
            ngx = 0; ngy = 0;
        }
        int done = 0;
        while (tgy != 0) {
            const unsigned ti = bfind(tgy);
            const uint32_t tri = tgx * 3u + ti * 3u;
            tgy &= ~(1u << ti);
            if ((uint64_t)tri + 3u > (uint64_t)woop_f4) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
            if (in_blas) {
                float t, u, v;
                if (woop_test(woop + tri, o, d, tmin, tmax, &t, &u, &v)) {
                    tmax = t; hit_addr = (int)tri; hit_inst = cur_inst; hu = u; hv = v;
                    if (any) { done = 1; break; }
                }
            } else {
                const int32_t inst = map[tri], b = map[tri + 1];
                if (b < 0 || b >= n_blas) { err |= ORACLE_ERR_BAD_SCENE; done = 1; break; }
                if (ngy > 0x00FFFFFFu) {
                    if (sp >= STACK_CAP) { err |= ORACLE_ERR_STACK; done = 1; break; }
                    stx[sp] = ngx; sty[sp] = ngy; ++sp;
                }
                if (tgy != 0) {
                    if (sp >= STACK_CAP) { err |= ORACLE_ERR_STACK; done = 1; break; }
                    stx[sp] = tgx; sty[sp] = tgy; ++sp;
                }
                inst_sp = sp; in_blas = 1; cur_inst = inst;
                const f4* r = woop + tri;
                const float oo[3] = {fmaf(r[0].z, wo[2], fmaf(r[0].y, wo[1], fmaf(r[0].x, wo[0], r[0].w))),
                                     fmaf(r[1].z, wo[2], fmaf(r[1].y, wo[1], fmaf(r[1].x, wo[0], r[1].w))),
                                     fmaf(r[2].z, wo[2], fmaf(r[2].y, wo[1], fmaf(r[2].x, wo[0], r[2].w)))};
                const float od[3] = {fmaf(r[0].z, wd[2], fmaf(r[0].y, wd[1], r[0].x * wd[0])),
                                     fmaf(r[1].z, wd[2], fmaf(r[1].y, wd[1], r[1].x * wd[0])),
                                     fmaf(r[2].z, wd[2], fmaf(r[2].y, wd[1], r[2].x * wd[0]))};
                SET_RAY(oo, od);
                nodes = (const f4*)bn[b]; node_f4 = bn_f4[b];
                woop = (const f4*)bw[b]; woop_f4 = bw_f4[b];
                ngx = 0; ngy = 0x80000000u; tgx = 0; tgy = 0;
                break;
            }
        }
        if (done) break;
        if (ngy <= 0x00FFFFFFu) {
            if (in_blas && sp == inst_sp) {
                in_blas = 0;
                nodes = tn; node_f4 = tn_f4; woop = rows; woop_f4 = rows_f4;
                SET_RAY(wo, wd);
            }
            if (sp > 0) { --sp; ngx = stx[sp]; ngy = sty[sp]; }
            else break;
        }
    }
#undef SET_RAY
    if (err) { hit_addr = -1; hit_inst = -1; }
    hit[0] = tmax; hit[1] = from_i(hit_addr); hit[2] = hu; hit[3] = hv;
    if (inst_out) *inst_out = hit_addr >= 0 ? hit_inst : -1;
    return err;
}

int oracle_trace_instanced(const float* tlas_nodes, int64_t tlas_node_f4, const float* tlas_rows, int64_t tlas_rows_f4,
                           const int32_t* tlas_map, int n_blas, const float* const* blas_nodes,
                           const int64_t* blas_node_f4, const float* const* blas_woop, const int64_t* blas_woop_f4,
                           const float* rays, int64_t n, int any_hit, float* hits, int32_t* inst_out, int threads) {
    int err = 0;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 256) reduction(| : err) num_threads(threads)
#endif
    for (int64_t i = 0; i < n; ++i)
        err |= inst_ray((const f4*)tlas_nodes, tlas_node_f4, (const f4*)tlas_rows, tlas_rows_f4, tlas_map, n_blas,
                        blas_nodes, blas_node_f4, blas_woop, blas_woop_f4, rays + 8 * i, any_hit, hits + 4 * i,
                        inst_out ? inst_out + i : NULL);
    (void)threads;
    return err;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void oracle_tri_f64(const float ray[8], const float v0[3], const float v1[3], const float v2[3], double out[4]) {
    double e0[3], e1[3], s[3], d[3];
    for (int a = 0; a < 3; ++a) {
        e0[a] = (double)v0[a] - v2[a];
        e1[a] = (double)v1[a] - v2[a];
        s[a] = (double)ray[a] - v2[a];
        d[a] = ray[4 + a];
    }
    /* Solve s = -t d + u e0 + v e1 by Cramer's rule on [e0 e1 -d]. */
    const double p[3] = {d[1] * e1[2] - d[2] * e1[1], d[2] * e1[0] - d[0] * e1[2], d[0] * e1[1] - d[1] * e1[0]};
    const double det = e0[0] * p[0] + e0[1] * p[1] + e0[2] * p[2];
    if (det == 0.0) {
        out[0] = INFINITY; out[1] = out[2] = NAN; out[3] = 0.0;
        return;
    }
    const double inv = 1.0 / det;
    const double u = (s[0] * p[0] + s[1] * p[1] + s[2] * p[2]) * inv;
    const double q[3] = {s[1] * e0[2] - s[2] * e0[1], s[2] * e0[0] - s[0] * e0[2], s[0] * e0[1] - s[1] * e0[0]};
    const double v = (d[0] * q[0] + d[1] * q[1] + d[2] * q[2]) * inv;
    const double t = (e1[0] * q[0] + e1[1] * q[1] + e1[2] * q[2]) * inv;
    out[0] = t; out[1] = u; out[2] = v; out[3] = det;
}

/* Philox4x32-10, Salmon et al., SC 2011. */
void oracle_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        c1 = (uint32_t)p1; c3 = (uint32_t)p0; c0 = n0; c2 = n2;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float unit24(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

/* src/ValidationKernels.cu:41-101 with the Philox stream in place of curand. */
void oracle_aorays(const float* pos, const float* nrm, const float* radius, int64_t n_surfels, int spp, uint64_t seed,
                   float tmin, float tmax, float offset_scale, float* out) {
    const int64_t n = n_surfels * spp;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < n; ++i) {
        const int64_t s = i / spp;
        const float p[3] = {pos[4 * s], pos[4 * s + 1], pos[4 * s + 2]};
        const float nn[3] = {nrm[4 * s], nrm[4 * s + 1], nrm[4 * s + 2]};
        const float r = radius ? radius[s] : 0.0f;
        if (nn[0] == 0.f && nn[1] == 0.f && nn[2] == 0.f) {  /* no surface: an empty ray */
            float* o = out + 8 * i;
            o[0] = p[0]; o[1] = p[1]; o[2] = p[2]; o[3] = 0.f;
            o[4] = 0.f; o[5] = 0.f; o[6] = 1.f; o[7] = 0.f;
            continue;
        }
        float t1[3] = {nn[1] * 1.0f - nn[2] * 0.0f, nn[2] * 0.0f - nn[0] * 1.0f, nn[0] * 0.0f - nn[1] * 0.0f};
        if (sqrtf(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]) < 0.1f) {
            t1[0] = nn[1] * 0.0f - nn[2] * 1.0f;
            t1[1] = nn[2] * 0.0f - nn[0] * 0.0f;
            t1[2] = nn[0] * 1.0f - nn[1] * 0.0f;
        }
        float l = sqrtf(t1[0] * t1[0] + t1[1] * t1[1] + t1[2] * t1[2]);
        for (int a = 0; a < 3; ++a) t1[a] = t1[a] * (1.0f / l);
        float t2[3] = {t1[1] * nn[2] - t1[2] * nn[1], t1[2] * nn[0] - t1[0] * nn[2], t1[0] * nn[1] - t1[1] * nn[0]};
        l = sqrtf(t2[0] * t2[0] + t2[1] * t2[1] + t2[2] * t2[2]);
        for (int a = 0; a < 3; ++a) t2[a] = t2[a] * (1.0f / l);
        const uint32_t ctr[4] = {(uint32_t)i, (uint32_t)((uint64_t)i >> 32), 0u, 0u};
        uint32_t rnd[4];
        oracle_philox(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), rnd);
        const float a = 2.0f * unit24(rnd[0]) - 1.0f, b = 2.0f * unit24(rnd[1]) - 1.0f;
        float x = 0.f, y = 0.f;
        if (a != 0.f || b != 0.f) {
            const float kPi = 3.1415926f;
            float rr, th;
            if (a * a > b * b) { rr = a; th = (kPi / 4.0f) * (b / a); }
            else { rr = b; th = (kPi / 2.0f) - (kPi / 4.0f) * (a / b); }
            x = rr * cosf(th);
            y = rr * sinf(th);
        }
        const float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
        float dd[3];
        for (int k = 0; k < 3; ++k) dd[k] = t1[k] * x + t2[k] * y + nn[k] * z;
        l = sqrtf(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
        float* o = out + 8 * i;
        for (int k = 0; k < 3; ++k) {
            o[k] = p[k] + nn[k] * (r * offset_scale);
            o[4 + k] = dd[k] * (1.0f / l);
        }
        o[3] = tmin;
        o[7] = tmax;
    }
}
