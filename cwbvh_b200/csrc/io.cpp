// Scene and sample-cache files.
//
// mesh.dat and samplecache.dat are the reference's input files, read by its
// main() (src/main.cpp:31-45 and :52-64): little-endian int32 counts followed
// by packed float3/int3/int32 (mesh) or float4/float4/float (sample cache)
// arrays.  The reference reads them without any check; here every count is
// checked against the file length and every index against the vertex count,
// so a short or corrupt file is an error, not an out-of-bounds read.
//
// A converted scene (the GPU-layout buffers of a host BVH) is stored in this
// library's own file format, so a resident scene can be reloaded without
// rebuilding:
//
//   offset  0  char[8]  "RQSCENE1"
//           8  uint32   kind (0 CWBVH, 1 BVH2)
//          12  int32    depth
//          16  int64    node float4s, Woop float4s, primitive-map entries,
//                       node count, leaf count
//          56  float[6] bounds lo xyz, hi xyz
//          80  uint64   FNV-1a 64 of the payload
//          88  payload  nodes (16 B each), Woop rows (16 B each), map (4 B each)
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <new>
#include <vector>

#include "host_common.h"

using namespace rq;

namespace {

struct File {
    std::FILE* f = nullptr;
    explicit File(const char* path, const char* mode) : f(std::fopen(path, mode)) {}
    ~File() {
        if (f) std::fclose(f);
    }
};

int64_t file_size(std::FILE* f) {
    if (std::fseek(f, 0, SEEK_END) != 0) return -1;
    const long n = std::ftell(f);
    if (std::fseek(f, 0, SEEK_SET) != 0) return -1;
    return (int64_t)n;
}

bool read_all(std::FILE* f, void* dst, int64_t bytes) {
    return bytes == 0 || std::fread(dst, 1, (size_t)bytes, f) == (size_t)bytes;
}

bool write_all(std::FILE* f, const void* src, int64_t bytes) {
    return bytes == 0 || std::fwrite(src, 1, (size_t)bytes, f) == (size_t)bytes;
}

template <class T>
T* alloc_array(int64_t n) {
    return static_cast<T*>(std::malloc((size_t)std::max<int64_t>(n, 1) * sizeof(T)));
}

uint64_t fnv1a(uint64_t h, const void* data, size_t bytes) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t k = 0; k < bytes; ++k) {
        h ^= p[k];
        h *= 0x100000001B3ull;
    }
    return h;
}

constexpr uint64_t kFnvBasis = 0xCBF29CE484222325ull;
constexpr char kSceneMagic[8] = {'R', 'Q', 'S', 'C', 'E', 'N', 'E', '1'};

#pragma pack(push, 1)
struct SceneHeader {
    char magic[8];
    uint32_t kind;
    int32_t depth;
    int64_t node_f4, woop_f4, prim_count, node_count, leaf_count;
    float bounds[6];
    uint64_t checksum;
};
#pragma pack(pop)
static_assert(sizeof(SceneHeader) == 88, "scene header layout");

uint64_t payload_checksum(const HostBVH& b) {
    uint64_t h = kFnvBasis;
    h = fnv1a(h, b.nodes.data(), b.nodes.size() * sizeof(float));
    h = fnv1a(h, b.woop.data(), b.woop.size() * sizeof(float));
    h = fnv1a(h, b.prim_index.data(), b.prim_index.size() * sizeof(int32_t));
    return h;
}

}  // namespace

extern "C" {

void rq_free_host(void* p) { std::free(p); }

rq_status rq_load_mesh_dat(const char* path, float** vertices, int64_t* nv, int32_t** indices, int64_t* nt,
                           int32_t** materials) {
    if (!path || !vertices || !nv || !indices || !nt) return RQ_ERR_INVALID_ARG;
    File file(path, "rb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const int64_t size = file_size(file.f);
    int32_t counts[2];
    if (size < 8 || !read_all(file.f, counts, 8)) return RQ_ERR_INVALID_ARG;
    const int64_t n_v = counts[0], n_t = counts[1];
    if (n_v < 0 || n_t < 0 || size != 8 + 12 * n_v + 16 * n_t) return RQ_ERR_INVALID_ARG;
    float* v = alloc_array<float>(3 * n_v);
    int32_t* i = alloc_array<int32_t>(3 * n_t);
    int32_t* m = alloc_array<int32_t>(n_t);
    if (!v || !i || !m) {
        std::free(v); std::free(i); std::free(m);
        return RQ_ERR_OOM;
    }
    bool ok = read_all(file.f, v, 12 * n_v) && read_all(file.f, i, 12 * n_t) && read_all(file.f, m, 4 * n_t);
    for (int64_t k = 0; ok && k < 3 * n_t; ++k) ok = i[k] >= 0 && i[k] < n_v;
    if (!ok) {
        std::free(v); std::free(i); std::free(m);
        return RQ_ERR_INVALID_ARG;
    }
    *vertices = v;
    *indices = i;
    *nv = n_v;
    *nt = n_t;
    if (materials) *materials = m;
    else std::free(m);
    return RQ_OK;
}

rq_status rq_save_mesh_dat(const char* path, const float* vertices, int64_t nv, const int32_t* indices, int64_t nt,
                           const int32_t* materials) {
    if (!path || nv < 0 || nt < 0 || nv > std::numeric_limits<int32_t>::max() ||
        nt > std::numeric_limits<int32_t>::max() || (nv > 0 && !vertices) || (nt > 0 && !indices))
        return RQ_ERR_INVALID_ARG;
    for (int64_t k = 0; k < 3 * nt; ++k)
        if (indices[k] < 0 || indices[k] >= nv) return RQ_ERR_INVALID_ARG;
    File file(path, "wb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const int32_t counts[2] = {(int32_t)nv, (int32_t)nt};
    bool ok = write_all(file.f, counts, 8) && write_all(file.f, vertices, 12 * nv) &&
              write_all(file.f, indices, 12 * nt);
    if (materials) {
        ok = ok && write_all(file.f, materials, 4 * nt);
    } else {
        const std::vector<int32_t> zeros((size_t)nt, 0);
        ok = ok && write_all(file.f, zeros.data(), 4 * nt);
    }
    return ok ? RQ_OK : RQ_ERR_INVALID_ARG;
}

rq_status rq_load_samplecache_dat(const char* path, int32_t* size_x, int32_t* size_y, float** pos, float** nrm,
                                  float** radius) {
    if (!path || !size_x || !size_y || !pos || !nrm || !radius) return RQ_ERR_INVALID_ARG;
    File file(path, "rb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const int64_t size = file_size(file.f);
    int32_t dims[2];
    if (size < 8 || !read_all(file.f, dims, 8)) return RQ_ERR_INVALID_ARG;
    if (dims[0] < 0 || dims[1] < 0) return RQ_ERR_INVALID_ARG;
    const int64_t n = (int64_t)dims[0] * dims[1];
    if (size != 8 + 36 * n) return RQ_ERR_INVALID_ARG;
    float* p = alloc_array<float>(4 * n);
    float* q = alloc_array<float>(4 * n);
    float* r = alloc_array<float>(n);
    if (!p || !q || !r) {
        std::free(p); std::free(q); std::free(r);
        return RQ_ERR_OOM;
    }
    if (!(read_all(file.f, p, 16 * n) && read_all(file.f, q, 16 * n) && read_all(file.f, r, 4 * n))) {
        std::free(p); std::free(q); std::free(r);
        return RQ_ERR_INVALID_ARG;
    }
    *size_x = dims[0];
    *size_y = dims[1];
    *pos = p;
    *nrm = q;
    *radius = r;
    return RQ_OK;
}

rq_status rq_save_samplecache_dat(const char* path, int32_t size_x, int32_t size_y, const float* pos,
                                  const float* nrm, const float* radius) {
    const int64_t n = (int64_t)size_x * size_y;
    if (!path || size_x < 0 || size_y < 0 || (n > 0 && (!pos || !nrm || !radius))) return RQ_ERR_INVALID_ARG;
    File file(path, "wb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const int32_t dims[2] = {size_x, size_y};
    const bool ok = write_all(file.f, dims, 8) && write_all(file.f, pos, 16 * n) && write_all(file.f, nrm, 16 * n) &&
                    write_all(file.f, radius, 4 * n);
    return ok ? RQ_OK : RQ_ERR_INVALID_ARG;
}

rq_status rq_host_bvh_save(rq_host_bvh_t bvh, const char* path) {
    if (!bvh || !path) return RQ_ERR_INVALID_ARG;
    const HostBVH& b = bvh->b;
    SceneHeader h{};
    std::memcpy(h.magic, kSceneMagic, 8);
    h.kind = (uint32_t)b.kind;
    h.depth = b.depth;
    h.node_f4 = (int64_t)b.nodes.size() / 4;
    h.woop_f4 = (int64_t)b.woop.size() / 4;
    h.prim_count = (int64_t)b.prim_index.size();
    h.node_count = b.node_count;
    h.leaf_count = b.leaf_count;
    const float bounds[6] = {b.bounds.lo.x, b.bounds.lo.y, b.bounds.lo.z, b.bounds.hi.x, b.bounds.hi.y, b.bounds.hi.z};
    std::memcpy(h.bounds, bounds, sizeof(bounds));
    h.checksum = payload_checksum(b);
    File file(path, "wb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const bool ok = write_all(file.f, &h, sizeof(h)) && write_all(file.f, b.nodes.data(), 16 * h.node_f4) &&
                    write_all(file.f, b.woop.data(), 16 * h.woop_f4) &&
                    write_all(file.f, b.prim_index.data(), 4 * h.prim_count);
    return ok ? RQ_OK : RQ_ERR_INVALID_ARG;
}

rq_status rq_host_bvh_load(const char* path, rq_host_bvh_t* out) {
    if (!path || !out) return RQ_ERR_INVALID_ARG;
    File file(path, "rb");
    if (!file.f) return RQ_ERR_NOT_FOUND;
    const int64_t size = file_size(file.f);
    SceneHeader h{};
    if (size < (int64_t)sizeof(h) || !read_all(file.f, &h, sizeof(h))) return RQ_ERR_BAD_SCENE;
    if (std::memcmp(h.magic, kSceneMagic, 8) != 0 || h.kind > 1u || h.node_f4 < 0 || h.woop_f4 < 0 ||
        h.prim_count != h.woop_f4 || h.node_count < 0 || h.leaf_count < 0 || h.depth < 0)
        return RQ_ERR_BAD_SCENE;
    const int64_t limit = std::numeric_limits<int64_t>::max() / 32;
    if (h.node_f4 > limit || h.woop_f4 > limit ||
        size != (int64_t)sizeof(h) + 16 * h.node_f4 + 16 * h.woop_f4 + 4 * h.prim_count)
        return RQ_ERR_BAD_SCENE;
    try {
        std::unique_ptr<rq_host_bvh> r(new rq_host_bvh());
        HostBVH& b = r->b;
        b.kind = (rq_bvh_kind)h.kind;
        b.depth = h.depth;
        b.node_count = h.node_count;
        b.leaf_count = h.leaf_count;
        b.bounds.lo = {h.bounds[0], h.bounds[1], h.bounds[2]};
        b.bounds.hi = {h.bounds[3], h.bounds[4], h.bounds[5]};
        b.has_tree = false;
        b.nodes.resize((size_t)(4 * h.node_f4));
        b.woop.resize((size_t)(4 * h.woop_f4));
        b.prim_index.resize((size_t)h.prim_count);
        if (!(read_all(file.f, b.nodes.data(), 16 * h.node_f4) && read_all(file.f, b.woop.data(), 16 * h.woop_f4) &&
              read_all(file.f, b.prim_index.data(), 4 * h.prim_count)))
            return RQ_ERR_BAD_SCENE;
        if (payload_checksum(b) != h.checksum) return RQ_ERR_BAD_SCENE;
        *out = r.release();
        return RQ_OK;
    } catch (const std::bad_alloc&) {
        return RQ_ERR_OOM;
    }
}

}  // extern "C"
