// Harness around the reference's own code, compiled from its sources by
// oracle/Makefile into oracle/_ref/libref.so.  TEST INFRASTRUCTURE ONLY: it
// gives the tests extern "C" access to
//   * ConvertToGPUBVH2 / ConvertToGPUCompressedWideBVH / WoopifyTriangle
//     (src/GPUBVHConverter.cpp:10-403), fed with this library's builder trees;
//   * rtBind*/rtTrace* (src/TraversalKernelCWBVH.cu:377-426,
//     src/TraversalKernelBVH2.cu:180-227), the reference's CUDA kernels, and
//     the CWBVH kernel launched with an occupancy-filling grid;
//   * GenerateAORaysUniform (src/ValidationKernels.cu:140-187).
// No reference source is copied here; they are compiled where they lie.
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "helper_math.h"
#include "EmbreeBVHBuilder.h"
#include "GPUBVHConverter.h"
#include "TraversalKernelBVH2.h"
#include "TraversalKernelCWBVH.h"
#include "ValidationKernels.h"

// The reference's persistent CWBVH kernel (defined in
// src/TraversalKernelCWBVH.cu, compiled in its own object).
__global__ void rtTraceCWBVHDynamicFetch(Ray* rayBuffer, Hit* rayResultBuffer, int rayCount, int* finishedRayCount);

namespace {

template <int W>
BVHNNode<W>* make_tree(int64_t node, const int32_t* codes, const float* boxes, const int32_t* leaf_first,
                       const int32_t* leaf_count, const int32_t* refs) {
    auto* n = new BVHNNode<W>();
    int count = 0;
    for (int c = 0; c < W; ++c) {
        const int32_t code = codes[node * W + c];
        if (code == -1) continue;
        const float* b = boxes + (node * W + c) * 6;
        n->ChildrenMin[count] = make_float3(b[0], b[1], b[2]);
        n->ChildrenMax[count] = make_float3(b[3], b[4], b[5]);
        if (code >= 0) {
            n->Children[count] = make_tree<W>(code, codes, boxes, leaf_first, leaf_count, refs);
        } else {
            const int32_t l = -code - 2;
            auto* leaf = new BVHNNode<W>();
            leaf->LeafPrimitiveCount = leaf_count[l];
            leaf->LeafPrimitiveRefs = new int[leaf_count[l]];
            for (int k = 0; k < leaf_count[l]; ++k) leaf->LeafPrimitiveRefs[k] = refs[leaf_first[l] + k];
            n->Children[count] = leaf;
        }
        ++count;
    }
    n->ChildCount = count;
    return n;
}

template <typename T>
T* export_vec(const std::vector<T>& v) {
    T* p = (T*)std::malloc(sizeof(T) * (v.size() ? v.size() : 1));
    if (!v.empty()) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

}  // namespace

extern "C" {

// Converts a builder tree with the reference converter.  The outputs are
// malloc'd (release with ref_free).  Woop rows come from the reference's
// WoopifyTriangle.
int ref_convert(int width, int64_t n_nodes, const int32_t* codes, const float* boxes, const int32_t* leaf_first,
                const int32_t* leaf_count, const int32_t* refs, int root_is_leaf, const float* verts,
                const int32_t* idx, float** out_nodes, int64_t* n_node_f4, float** out_woop, int64_t* n_woop_f4,
                int32_t** out_prim, int64_t* n_prim) {
    auto append = [&](int prim, std::vector<float4>& out) {
        float4 v0, v1, v2;
        const int32_t* t = idx + 3 * (int64_t)prim;
        WoopifyTriangle(make_float3(verts[3 * t[0]], verts[3 * t[0] + 1], verts[3 * t[0] + 2]),
                        make_float3(verts[3 * t[1]], verts[3 * t[1] + 1], verts[3 * t[1] + 2]),
                        make_float3(verts[3 * t[2]], verts[3 * t[2] + 1], verts[3 * t[2] + 2]), v0, v1, v2);
        out.push_back(v0);
        out.push_back(v1);
        out.push_back(v2);
    };
    GPUBVHIntermediates out;
    if (width == 2) {
        BVH2Node* root;
        if (root_is_leaf) {
            root = new BVH2Node();
            root->LeafPrimitiveCount = leaf_count[0];
            root->LeafPrimitiveRefs = new int[leaf_count[0] > 0 ? leaf_count[0] : 1];
            for (int k = 0; k < leaf_count[0]; ++k) root->LeafPrimitiveRefs[k] = refs[leaf_first[0] + k];
        } else {
            root = make_tree<2>(0, codes, boxes, leaf_first, leaf_count, refs);
        }
        ConvertToGPUBVH2(root, append, out);
        root->Release();
        delete root;
    } else if (width == 8) {
        if (n_nodes <= 0) return 1;
        BVH8Node* root = make_tree<8>(0, codes, boxes, leaf_first, leaf_count, refs);
        ConvertToGPUCompressedWideBVH(root, append, out);
        root->Release();
        delete root;
    } else {
        return 1;
    }
    *out_nodes = (float*)export_vec(out.BVHNodeData);
    *n_node_f4 = (int64_t)out.BVHNodeData.size();
    *out_woop = (float*)export_vec(out.InlinedPrimitives);
    *n_woop_f4 = (int64_t)out.InlinedPrimitives.size();
    *out_prim = export_vec(out.PrimitiveIndices);
    *n_prim = (int64_t)out.PrimitiveIndices.size();
    return 0;
}

void ref_free(void* p) { std::free(p); }

void ref_woopify(const float* v0, const float* v1, const float* v2, float* out12) {
    float4 a, b, c;
    WoopifyTriangle(make_float3(v0[0], v0[1], v0[2]), make_float3(v1[0], v1[1], v1[2]),
                    make_float3(v2[0], v2[1], v2[2]), a, b, c);
    std::memcpy(out12, &a, 16);
    std::memcpy(out12 + 4, &b, 16);
    std::memcpy(out12 + 8, &c, 16);
}

// Reference kernels (GPU only).  Pointers are device pointers.
void ref_bind_cwbvh(const void* nodes, const void* woop, const int32_t* prim) {
    rtBindCWBVHData((const float4*)nodes, (const float4*)woop, prim);
}
void ref_trace_cwbvh(void* rays, void* hits, int n) { rtTraceCWBVH((Ray*)rays, (Hit*)hits, n); }
void ref_bind_bvh2(const void* nodes, const void* woop, const int32_t* prim) {
    rtBindBVH2Data((const float4*)nodes, (const float4*)woop, prim);
}
void ref_trace_bvh2(void* rays, void* hits, int n) { rtTraceBVH2((Ray*)rays, (Hit*)hits, n); }

// The reference's CWBVH kernel itself (src/TraversalKernelCWBVH.cu:24-29: its
// blocks are 32 x 2 threads, its grid persistent with a global ray counter),
// launched with `blocks` blocks instead of rtTraceCWBVH's fixed 32 x 32
// (src/TraversalKernelCWBVH.cu:401-402), on the legacy default stream like
// rtTraceCWBVH.  blocks <= 0: as many as are resident at once on the device
// (occupancy-filling).  `counter` is a device int the call zeroes first.
// Returns the CUDA error code of the launch (the caller waits for it);
// *used_blocks receives the grid size.
int ref_trace_cwbvh_grid(void* rays, void* hits, int n, int blocks, int* counter, int* used_blocks) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rtTraceCWBVHDynamicFetch, 64, 0);
    if (e != cudaSuccess) return (int)e;
    if (blocks <= 0) blocks = sms * (per_sm > 0 ? per_sm : 1);
    if (used_blocks) *used_blocks = blocks;
    e = cudaMemsetAsync(counter, 0, sizeof(int), 0);
    if (e == cudaSuccess) {
        rtTraceCWBVHDynamicFetch<<<blocks, dim3(32, 2)>>>((Ray*)rays, (Hit*)hits, n, counter);
        e = cudaGetLastError();
    }
    return (int)e;
}

// Reference AO ray generation (curand XORWOW); returns a device buffer owned
// by the caller (cudaFree).
void* ref_aorays(int n, int spp, float* pos, float* nrm, float* radius) {
    return GenerateAORaysUniform(n, spp, (float4*)pos, (float4*)nrm, radius);
}

int ref_cuda_free(void* p) { return (int)cudaFree(p); }
int ref_sync(void) { return (int)cudaDeviceSynchronize(); }

}  // extern "C"
