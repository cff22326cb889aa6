// AO ray generation from a surfel sample cache, surfel sampling on triangles,
// the per-surfel AO reduction and Morton ray sorting.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>

#include "runtime.h"
#include "trace_common.cuh"

namespace rq {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As
// Easy as 1, 2, 3", SC 2011): a counter-based generator, so ray i's numbers
// depend only on (seed, i) and any thread can make them.
struct U4 {
    uint32_t x, y, z, w;
};
__host__ __device__ inline U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)M0 * c.x;
        const uint64_t p1 = (uint64_t)M1 * c.z;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}
// Uniform in (0, 1] from the top 24 bits (curand_uniform's range).
__host__ __device__ inline float unit24(uint32_t r) { return (float)((r >> 8) + 1u) * (1.0f / 16777216.0f); }

__device__ inline float3 f3(float4 v) { return make_float3(v.x, v.y, v.z); }
__device__ inline float3 add3(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ inline float3 mul3(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
__device__ inline float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ inline float len3(float3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ inline float3 norm3(float3 a) { return mul3(a, 1.0f / len3(a)); }

// One ray per (surfel, sample), surfel = i / spp: tangent frame from n x z
// (n x y when that is short), concentric disk lifted to the cosine
// hemisphere, origin pushed off the surface by radius * offset_scale
// (src/ValidationKernels.cu:41-101).  The random stream of ray i is keyed by
// its index first_ray + i in the whole request, so a request generated in
// pieces gives the same rays as in one call.
__global__ void aorays_kernel(const float4* __restrict__ pos, const float4* __restrict__ nrm,
                              const float* __restrict__ radius, int64_t n_rays, int spp, int64_t first_ray,
                              uint32_t k0, uint32_t k1, float tmin, float tmax, float offset_scale,
                              Ray* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rays) return;
    const int64_t s = i / spp;
    const float3 p = f3(pos[s]);
    const float3 n = f3(nrm[s]);
    const float r = radius ? radius[s] : 0.0f;
    if (n.x == 0.f && n.y == 0.f && n.z == 0.f) {  // no surface (a primary miss): an empty ray
        out[i].origin_tmin = make_float4(p.x, p.y, p.z, 0.f);
        out[i].dir_tmax = make_float4(0.f, 0.f, 1.f, 0.f);
        return;
    }
    float3 t1 = cross3(n, make_float3(0.f, 0.f, 1.f));
    if (len3(t1) < 0.1f) t1 = cross3(n, make_float3(0.f, 1.f, 0.f));
    t1 = norm3(t1);
    const float3 t2 = norm3(cross3(t1, n));
    const uint64_t ctr = (uint64_t)(first_ray + i);
    const U4 rnd = philox4x32_10(U4{(uint32_t)ctr, (uint32_t)(ctr >> 32), 0u, 0u}, k0, k1);
    const float a = 2.0f * unit24(rnd.x) - 1.0f, b = 2.0f * unit24(rnd.y) - 1.0f;
    float dxl = 0.f, dyl = 0.f;
    if (a != 0.f || b != 0.f) {
        const float kPi = 3.1415926f;
        float rr, th;
        if (a * a > b * b) {
            rr = a;
            th = (kPi / 4.0f) * (b / a);
        } else {
            rr = b;
            th = (kPi / 2.0f) - (kPi / 4.0f) * (a / b);
        }
        dxl = rr * cosf(th);
        dyl = rr * sinf(th);
    }
    const float dzl = sqrtf(fmaxf(0.0f, 1.0f - dxl * dxl - dyl * dyl));
    const float3 d = norm3(add3(add3(mul3(t1, dxl), mul3(t2, dyl)), mul3(n, dzl)));
    const float3 o = add3(p, mul3(n, r * offset_scale));
    out[i].origin_tmin = make_float4(o.x, o.y, o.z, tmin);
    out[i].dir_tmax = make_float4(d.x, d.y, d.z, tmax);
}

// Surfel i on triangle floor(u * nt) at barycentrics (1 - sqrt(a), b sqrt(a)).
__global__ void surfels_kernel(const float* __restrict__ v, const int32_t* __restrict__ idx, int64_t nt,
                               int64_t n, uint32_t k0, uint32_t k1, float4* __restrict__ pos,
                               float4* __restrict__ nrm, float* __restrict__ radius) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const U4 rnd = philox4x32_10(U4{(uint32_t)i, (uint32_t)((uint64_t)i >> 32), 1u, 0u}, k0, k1);
    const uint64_t pick = ((uint64_t)rnd.x << 32 | rnd.y);
    const int64_t t = (int64_t)(((unsigned __int128)pick * (unsigned __int128)nt) >> 64);
    const float su = sqrtf(unit24(rnd.z)), bv = unit24(rnd.w);
    const float b0 = 1.0f - su, b1 = bv * su, b2 = 1.0f - b0 - b1;
    const int32_t* tri = idx + 3 * t;
    const float3 p0 = make_float3(v[3 * tri[0]], v[3 * tri[0] + 1], v[3 * tri[0] + 2]);
    const float3 p1 = make_float3(v[3 * tri[1]], v[3 * tri[1] + 1], v[3 * tri[1] + 2]);
    const float3 p2 = make_float3(v[3 * tri[2]], v[3 * tri[2] + 1], v[3 * tri[2] + 2]);
    const float3 p = add3(add3(mul3(p0, b0), mul3(p1, b1)), mul3(p2, b2));
    const float3 nn = norm3(cross3(sub3(p1, p0), sub3(p2, p0)));
    pos[i] = make_float4(p.x, p.y, p.z, 1.0f);
    nrm[i] = make_float4(nn.x, nn.y, nn.z, 0.0f);
    if (radius) radius[i] = 0.0f;
}

// Pinhole camera: pixel (x, y) centre through an image plane at distance 1.
// Ray i is pixel (x, y) of tile i / (tw * th), tiles row-major across the
// image and pixels row-major within a tile (tw = width, th = 1: the image
// row-major).
__global__ void camera_rays_kernel(float3 eye, float3 fwd, float3 right, float3 upv, float half_w, float half_h,
                                   int width, int height, int tw, int th, float tmin, float tmax,
                                   Ray* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)width * height) return;
    const int64_t tile = i / ((int64_t)tw * th);
    const int in_tile = (int)(i % ((int64_t)tw * th));
    const int tiles_x = width / tw;
    const int x = (int)(tile % tiles_x) * tw + in_tile % tw;
    const int y = (int)(tile / tiles_x) * th + in_tile / tw;
    const float sx = ((x + 0.5f) / width * 2.0f - 1.0f) * half_w;
    const float sy = (1.0f - (y + 0.5f) / height * 2.0f) * half_h;
    const float3 d = norm3(add3(add3(fwd, mul3(right, sx)), mul3(upv, sy)));
    out[i].origin_tmin = make_float4(eye.x, eye.y, eye.z, tmin);
    out[i].dir_tmax = make_float4(d.x, d.y, d.z, tmax);
}

// Hit point and facing geometric normal of each closest hit.
__global__ void surfels_from_hits_kernel(const Ray* __restrict__ rays, const Hit* __restrict__ hits,
                                         const float4* __restrict__ woop, int64_t woop_f4, int64_t n,
                                         float4* __restrict__ pos, float4* __restrict__ nrm,
                                         float* __restrict__ radius) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 o = rays[i].origin_tmin, d = rays[i].dir_tmax;
    const float4 h = hits[i].t_triId_u_v;
    const int addr = __float_as_int(h.y);
    if (addr < 0 || addr >= woop_f4) {
        pos[i] = make_float4(o.x, o.y, o.z, 1.0f);
        nrm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    } else {
        const float4 v0 = __ldg(woop + addr);  // V0 = triangle-space z row: normal to the triangle
        float3 nn = norm3(make_float3(v0.x, v0.y, v0.z));
        if (nn.x * d.x + nn.y * d.y + nn.z * d.z > 0.f) nn = mul3(nn, -1.0f);
        pos[i] = make_float4(o.x + h.x * d.x, o.y + h.x * d.y, o.z + h.x * d.z, 1.0f);
        nrm[i] = make_float4(nn.x, nn.y, nn.z, 0.f);
    }
    if (radius) radius[i] = 0.0f;
}

// Fraction of a surfel's spp rays whose hit id is not -1.
__global__ void ao_reduce_kernel(const Hit* __restrict__ hits, int64_t n_surfels, int spp, float* __restrict__ ao) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_surfels) return;
    int occ = 0;
    for (int k = 0; k < spp; ++k) occ += __float_as_int(hits[s * spp + k].t_triId_u_v.y) != -1;
    ao[s] = (float)occ / (float)spp;
}

// ----------------------------------------------------------------- sorting

__device__ inline uint32_t spread10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// 32-bit ray key: 3 x 9-bit Morton code of the origin inside the item's
// bounds (high 27 bits) then the direction octant (low 3 bits); the item
// number sits above it so every item's rays stay together.
__global__ void morton_keys_kernel(const TraceItem* __restrict__ items, int n_items, const float* __restrict__ bounds,
                                   int64_t total, uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].ray_begin <= g) lo = mid; else hi = mid - 1;
    }
    const TraceItem& it = items[lo];
    const int64_t k = g - it.ray_begin;
    const float4 o = it.rays[k].origin_tmin;
    const float4 d = it.rays[k].dir_tmax;
    const float* b = bounds + 6 * lo;
    uint32_t q[3];
    const float oo[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ext = b[3 + a] - b[a];
        float f = ext > 0.f ? (oo[a] - b[a]) / ext : 0.f;
        f = fminf(fmaxf(f, 0.f), 1.f);
        q[a] = min(511u, (uint32_t)(f * 512.0f));
    }
    const uint32_t m = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    const uint32_t oct = (d.x < 0.f ? 4u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 1u : 0u);
    keys[g] = ((uint64_t)lo << 32) | ((uint64_t)m << 3) | oct;
    vals[g] = (int32_t)k;
}

__global__ void gather_rays_kernel(const TraceItem* __restrict__ items, const uint64_t* __restrict__ keys,
                                   const int32_t* __restrict__ vals, int64_t total, Ray* __restrict__ sorted) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total) return;
    const int item = (int)(keys[g] >> 32);
    const Ray* src = items[item].rays + vals[g];
    sorted[g].origin_tmin = __ldg(&src->origin_tmin);
    sorted[g].dir_tmax = __ldg(&src->dir_tmax);
}

static unsigned blocks_for(int64_t n, int b) { return (unsigned)((n + b - 1) / b); }

rq_status aorays_launch(const float* pos, const float* nrm, const float* radius, int64_t n_surfels, int spp,
                        int64_t first_ray, uint64_t seed, float tmin, float tmax, float offset_scale, rq_ray* out_rays,
                        void* stream) {
    if (n_surfels < 0 || spp <= 0 || first_ray < 0 || (n_surfels > 0 && (!pos || !nrm || !out_rays)))
        return RQ_ERR_INVALID_ARG;
    const int64_t n = n_surfels * spp;
    if (n == 0) return RQ_OK;
    aorays_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        (const float4*)pos, (const float4*)nrm, radius, n, spp, first_ray, (uint32_t)seed, (uint32_t)(seed >> 32),
        tmin, tmax, offset_scale, (Ray*)out_rays);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

rq_status sort_plan_create(const std::vector<TraceItem>& items, const std::vector<float>& bounds, SortPlan& plan) {
    plan = SortPlan();
    plan.n_items = (int)items.size();
    std::vector<TraceItem> src = items;
    int64_t off = 0;
    for (auto& it : src) {
        it.ray_begin = off;
        off += it.count;
    }
    plan.total = off;
    int bits = 1;
    while ((1 << bits) < plan.n_items) ++bits;
    plan.end_bit = 32 + bits;
    if (plan.total == 0) return RQ_OK;
    const size_t n = (size_t)plan.total;
    RQ_CUDA(cudaMalloc(&plan.keys_in, n * 8));
    RQ_CUDA(cudaMalloc(&plan.keys_out, n * 8));
    RQ_CUDA(cudaMalloc(&plan.vals_in, n * 4));
    RQ_CUDA(cudaMalloc(&plan.vals_out, n * 4));
    RQ_CUDA(cudaMalloc(&plan.sorted, n * sizeof(Ray)));
    RQ_CUDA(cudaMalloc(&plan.src_items, src.size() * sizeof(TraceItem)));
    RQ_CUDA(cudaMemcpy(plan.src_items, src.data(), src.size() * sizeof(TraceItem), cudaMemcpyHostToDevice));
    RQ_CUDA(cudaMalloc(&plan.bounds, bounds.size() * sizeof(float)));
    RQ_CUDA(cudaMemcpy(plan.bounds, bounds.data(), bounds.size() * sizeof(float), cudaMemcpyHostToDevice));
    RQ_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, plan.cub_temp_bytes, plan.keys_in, plan.keys_out, plan.vals_in,
                                            plan.vals_out, (int64_t)n, 0, plan.end_bit));
    RQ_CUDA(cudaMalloc(&plan.cub_temp, std::max<size_t>(16, plan.cub_temp_bytes)));
    // Count the kernels of one sort by capturing it once (not executed).
    cudaStream_t cs;
    RQ_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
        sort_plan_run(plan, cs);
        if (cudaStreamEndCapture(cs, &g) == cudaSuccess && g) {
            size_t n = 0;
            cudaGraphGetNodes(g, nullptr, &n);
            std::vector<cudaGraphNode_t> nodes(n);
            cudaGraphGetNodes(g, nodes.data(), &n);
            for (auto nd : nodes) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++plan.n_kernels;
            }
            cudaGraphDestroy(g);
        }
    }
    cudaGetLastError();
    cudaStreamDestroy(cs);
    return RQ_OK;
}

int sort_plan_kernel_count(const SortPlan& plan) { return plan.n_kernels; }

rq_status sort_plan_run(SortPlan& plan, cudaStream_t s) {
    if (plan.total == 0) return RQ_OK;
    morton_keys_kernel<<<blocks_for(plan.total, 256), 256, 0, s>>>(plan.src_items, plan.n_items, plan.bounds,
                                                                   plan.total, plan.keys_in, plan.vals_in);
    RQ_CUDA(cudaGetLastError());
    size_t tb = plan.cub_temp_bytes;
    RQ_CUDA(cub::DeviceRadixSort::SortPairs(plan.cub_temp, tb, plan.keys_in, plan.keys_out, plan.vals_in,
                                            plan.vals_out, plan.total, 0, plan.end_bit, s));
    gather_rays_kernel<<<blocks_for(plan.total, 256), 256, 0, s>>>(plan.src_items, plan.keys_out, plan.vals_out,
                                                                   plan.total, plan.sorted);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

void sort_plan_destroy(SortPlan& plan) {
    cudaFree(plan.keys_in);
    cudaFree(plan.keys_out);
    cudaFree(plan.vals_in);
    cudaFree(plan.vals_out);
    cudaFree(plan.sorted);
    cudaFree(plan.src_items);
    cudaFree(plan.bounds);
    cudaFree(plan.cub_temp);
    plan = SortPlan();
}

}  // namespace rq

using namespace rq;

extern "C" {

rq_status rq_aorays(const float* pos, const float* nrm, const float* radius, int64_t n_surfels, int spp, uint64_t seed,
                    float tmin, float tmax, float offset_scale, rq_ray* out_rays, void* stream) {
    return rq::aorays_launch(pos, nrm, radius, n_surfels, spp, 0, seed, tmin, tmax, offset_scale, out_rays, stream);
}

rq_status rq_sample_surfels(const float* vertices, const int32_t* indices, int64_t nt, int64_t n_surfels,
                            uint64_t seed, float* out_pos, float* out_nrm, float* out_radius, void* stream) {
    if (nt <= 0 || n_surfels < 0 || !vertices || !indices || (n_surfels > 0 && (!out_pos || !out_nrm)))
        return RQ_ERR_INVALID_ARG;
    if (n_surfels == 0) return RQ_OK;
    surfels_kernel<<<blocks_for(n_surfels, 256), 256, 0, (cudaStream_t)stream>>>(
        vertices, indices, nt, n_surfels, (uint32_t)seed, (uint32_t)(seed >> 32), (float4*)out_pos, (float4*)out_nrm,
        out_radius);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

static rq_status camera_rays_impl(const float eye[3], const float look[3], const float up[3], float vfov_deg,
                                  int width, int height, int tw, int th, float tmin, float tmax, rq_ray* out_rays,
                                  void* stream) {
    if (!eye || !look || !up || width <= 0 || height <= 0 || !(vfov_deg > 0.f && vfov_deg < 180.f) || !out_rays)
        return RQ_ERR_INVALID_ARG;
    if (tw <= 0 || th <= 0 || width % tw != 0 || height % th != 0) return RQ_ERR_INVALID_ARG;
    // Camera frame on the host (once per call).
    auto norm = [](float3 a) {
        const float l = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        return make_float3(a.x / l, a.y / l, a.z / l);
    };
    auto cross = [](float3 a, float3 b) {
        return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
    };
    auto len = [](float3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); };
    const float3 e = make_float3(eye[0], eye[1], eye[2]);
    const float3 view = make_float3(look[0] - eye[0], look[1] - eye[1], look[2] - eye[2]);
    if (!(len(view) > 0.f) || !std::isfinite(len(view))) return RQ_ERR_INVALID_ARG;
    const float3 fwd = norm(view);
    const float3 side = cross(fwd, make_float3(up[0], up[1], up[2]));
    if (!(len(side) > 1e-6f) || !std::isfinite(len(side))) return RQ_ERR_INVALID_ARG;  // up parallel to the view
    const float3 right = norm(side);
    const float3 upv = cross(right, fwd);
    const float half_h = std::tan(vfov_deg * 0.5f * 3.14159265358979f / 180.0f);
    const float half_w = half_h * (float)width / (float)height;
    const int64_t n = (int64_t)width * height;
    camera_rays_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(e, fwd, right, upv, half_w, half_h, width,
                                                                             height, tw, th, tmin, tmax,
                                                                             (Ray*)out_rays);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

rq_status rq_camera_rays(const float eye[3], const float look[3], const float up[3], float vfov_deg, int width,
                         int height, float tmin, float tmax, rq_ray* out_rays, void* stream) {
    return camera_rays_impl(eye, look, up, vfov_deg, width, height, width, 1, tmin, tmax, out_rays, stream);
}

rq_status rq_camera_rays_tiled(const float eye[3], const float look[3], const float up[3], float vfov_deg,
                               int width, int height, int tile_w, int tile_h, float tmin, float tmax,
                               rq_ray* out_rays, void* stream) {
    return camera_rays_impl(eye, look, up, vfov_deg, width, height, tile_w, tile_h, tmin, tmax, out_rays, stream);
}

rq_status rq_surfels_from_hits(rq_scene_t scene, const rq_ray* rays, const rq_hit* hits, int64_t count,
                               float* out_pos, float* out_nrm, float* out_radius, void* stream) {
    if (!scene || count < 0 || (count > 0 && (!rays || !hits || !out_pos || !out_nrm))) return RQ_ERR_INVALID_ARG;
    if (count == 0) return RQ_OK;
    surfels_from_hits_kernel<<<blocks_for(count, 256), 256, 0, (cudaStream_t)stream>>>(
        (const Ray*)rays, (const Hit*)hits, scene->woop, scene->woop_f4, count, (float4*)out_pos, (float4*)out_nrm,
        out_radius);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

rq_status rq_ao_reduce(const rq_hit* hits, int64_t n_surfels, int spp, float* out_ao, void* stream) {
    if (n_surfels < 0 || spp <= 0 || (n_surfels > 0 && (!hits || !out_ao))) return RQ_ERR_INVALID_ARG;
    if (n_surfels == 0) return RQ_OK;
    ao_reduce_kernel<<<blocks_for(n_surfels, 256), 256, 0, (cudaStream_t)stream>>>((const Hit*)hits, n_surfels, spp,
                                                                                   out_ao);
    RQ_CUDA(cudaGetLastError());
    return RQ_OK;
}

rq_status rq_sort_rays(rq_ctx_t ctx, const rq_ray* rays, int64_t count, const float bounds_lo[3],
                       const float bounds_hi[3], rq_ray* sorted_rays, int32_t* perm, void* stream) {
    if (!ctx || count < 0 || (count > 0 && (!rays || !sorted_rays || !perm || !bounds_lo || !bounds_hi)))
        return RQ_ERR_INVALID_ARG;
    if (count == 0) return RQ_OK;
    cudaStream_t s = (cudaStream_t)stream;
    TraceItem it{};
    it.rays = (const Ray*)rays;
    it.count = count;
    SortPlan plan;
    std::vector<float> b = {bounds_lo[0], bounds_lo[1], bounds_lo[2], bounds_hi[0], bounds_hi[1], bounds_hi[2]};
    rq_status st = sort_plan_create({it}, b, plan);
    if (st == RQ_OK) st = sort_plan_run(plan, s);
    if (st == RQ_OK) {
        cudaError_t e = cudaMemcpyAsync(sorted_rays, plan.sorted, (size_t)count * sizeof(Ray), cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(perm, plan.vals_out, (size_t)count * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "rq_sort_rays");
    }
    sort_plan_destroy(plan);
    return st;
}

}  // extern "C"
