/*
 * rq.h -- C ABI of the B200 ray-query engine (librq.so).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and returns
 * an rq_status (the reference aborts through cudaCheck/assert instead,
 * src/CUDAAssert.h:5-12).  Device pointers are raw CUDA device addresses;
 * streams are cudaStream_t handles passed as void*.
 *
 * Byte layouts kept from the reference (the drop-in contract):
 *   Ray  = { float4 origin_tmin; float4 dir_tmax; }   32 B  (src/helper_math.h:1853-1857)
 *   Hit  = { float4 t_triId_u_v; }                    16 B  (src/helper_math.h:1859-1865)
 *          y holds the int bits of the Woop float4 address of the hit
 *          triangle, or -1 for a miss.
 *   CWBVH node = 5 x float4 = 80 B                    (src/GPUBVHConverter.cpp:141-145,310-375)
 *   BVH2 node  = 4 x float4 = 64 B                    (src/GPUBVHConverter.cpp:69-72)
 *   Woop triangle = 3 x float4 = 48 B                 (src/GPUBVHConverter.cpp:380-403)
 *   BVH2 leaves end with a float4 whose x bits are 0x80000000
 *                                                     (src/GPUBVHConverter.cpp:116-117)
 */
#ifndef RQ_H
#define RQ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */

typedef enum rq_status {
    RQ_OK = 0,
    RQ_ERR_INVALID_ARG = 1,     /* null pointer, negative count, bad enum     */
    RQ_ERR_OOM = 2,             /* device or host allocation failed          */
    RQ_ERR_STACK_OVERFLOW = 3,  /* a ray needed more traversal stack entries  */
    RQ_ERR_TIMEOUT = 4,         /* a ray exceeded its traversal step budget  */
    RQ_ERR_CUDA = 5,            /* a CUDA runtime call failed                */
    RQ_ERR_BAD_SCENE = 6,       /* a node/triangle index left the buffers    */
    RQ_ERR_NOT_FOUND = 7,       /* unknown scene / request / ticket           */
    RQ_ERR_BUDGET = 8,          /* request larger than the server HBM budget  */
    RQ_ERR_CANCELLED = 9,       /* request cancelled or server shut down      */
    RQ_ERR_NO_DEVICE = 10       /* no CUDA device visible                    */
} rq_status;

/* Human-readable name of a status code (static storage). */
const char* rq_status_string(rq_status s);

/* Text of the last CUDA error seen by this thread (static per-thread storage). */
const char* rq_last_error(void);

/* ------------------------------------------------------------------- types */

typedef struct rq_ray { float origin_tmin[4]; float dir_tmax[4]; } rq_ray;
typedef struct rq_hit { float t_triId_u_v[4]; } rq_hit;

typedef enum rq_bvh_kind { RQ_BVH_CWBVH = 0, RQ_BVH_BVH2 = 1 } rq_bvh_kind;
typedef enum rq_query { RQ_CLOSEST = 0, RQ_ANY = 1 } rq_query;

/* Launch parameters of the persistent trace kernels.  Zero fields take the
 * built-in defaults (or the autotuner's cached choice, see rq_autotune). */
typedef struct rq_launch {
    int block_size;       /* threads per block: 64, 128, 256 or 512             */
    int blocks_per_sm;    /* persistent grid = SMs x this (0 = occupancy max)   */
    int smem_stack;       /* stack entries per lane in shared memory: 4, 8, 16  */
    float postpone_ratio; /* triangle postponing threshold Rt (reference 0.2)   */
    int fetch_nd;         /* dynamic fetch: idle lanes tolerated per iteration (default 2,      */
                          /* reference 4; negative = 0)                                          */
    int fetch_nw;         /* dynamic fetch: lost-lane budget before a refill (default 8, ref. 16) */
    int step_limit;       /* node visits per ray before it ends with RQ_ERR_TIMEOUT (0 = 2^22) */
} rq_launch;

/* --------------------------------------------------- host BVH construction */
/*
 * A host BVH is the converter output of the reference: node buffer, Woop
 * triangle buffer and the Woop-address -> primitive-index map, laid out
 * byte-for-byte as ConvertToGPUBVH2 / ConvertToGPUCompressedWideBVH emit them
 * (src/GPUBVHConverter.h:6-32).  The topology comes from this library's own
 * binned-SAH builder, which replaces BuildBVH2Triangle / BuildBVH8Triangle
 * (src/EmbreeBVHBuilder.h:39-43; Embree is not used).
 */
typedef struct rq_host_bvh* rq_host_bvh_t;

typedef struct rq_build_params {
    int max_leaf_size;    /* BVH2: max triangles per leaf (default 4); CWBVH is fixed at 3 */
    int sah_bins;         /* binned-SAH bins per axis (default 32)                         */
    int max_depth;        /* BVH2 depth limit (default 30; the reference stack is 32)      */
    int threads;          /* builder threads (0 = hardware concurrency)                    */
    int presplit;         /* 1, 2, 4 or 8: cut badly fitting triangles into up to this     */
                          /* many references with clipped boxes before the build (0 = 1)   */
    int treelet_passes;   /* passes of SAH treelet restructuring of the binary tree (CWBVH: */
                          /* before the 8-wide collapse; BVH2: kept if the depth stays     */
                          /* within max_depth) (0 = default 4, negative = none)            */
    int spatial_splits;   /* binned spatial splits in the SAH build (as Embree's high-     */
                          /* quality builder): budget of duplicate triangle references in  */
                          /* percent of the triangle count (0 = default 200, negative = none) */
} rq_build_params;

typedef struct rq_bvh_info {
    int64_t node_float4s;     /* length of the node buffer in float4          */
    int64_t woop_float4s;     /* length of the Woop buffer in float4          */
    int64_t prim_index_count; /* length of the Woop-address -> primitive map  */
    int64_t node_count;       /* nodes (80 B CWBVH / 64 B BVH2)              */
    int64_t leaf_count;
    int32_t depth;            /* levels from root to the deepest leaf          */
    int32_t kind;             /* rq_bvh_kind                                   */
    float bounds_lo[3];
    float bounds_hi[3];
} rq_bvh_info;

/* Build a BVH over an indexed triangle mesh (vertices: 3*nv floats, indices:
 * 3*nt ints) and convert it to the GPU layout of `kind`. */
rq_status rq_build_bvh(const float* vertices, int64_t nv, const int32_t* indices, int64_t nt,
                       rq_bvh_kind kind, const rq_build_params* params, rq_host_bvh_t* out);
rq_status rq_host_bvh_info(rq_host_bvh_t bvh, rq_bvh_info* out);
/* Borrowed pointers into the host BVH (valid until rq_host_bvh_free). */
rq_status rq_host_bvh_buffers(rq_host_bvh_t bvh, const float** nodes, const float** woop,
                              const int32_t** prim_index);
void rq_host_bvh_free(rq_host_bvh_t bvh);

/* The builder's tree before conversion, for checking the converter against
 * the reference's (src/GPUBVHConverter.cpp:10-378 consumes the same
 * BVHNNode<N> shape, src/EmbreeBVHBuilder.h:7-37).  width is 2 (BVH2) or 8
 * (CWBVH).  Per node: `width` child codes (>= 0 inner node, -1 empty slot,
 * <= -2 leaf number -(code+2)) and `width` child boxes (lo xyz, hi xyz).
 * Per leaf: first index into prim_refs and count.  Call with null arrays to
 * get the sizes, then with arrays of those sizes. */
rq_status rq_host_bvh_tree(rq_host_bvh_t bvh, int32_t* width, int64_t* n_nodes, int64_t* n_leaves,
                           int64_t* n_prim_refs, int32_t* root_is_leaf, int32_t* child_codes,
                           float* child_boxes, int32_t* leaf_first, int32_t* leaf_count,
                           int32_t* prim_refs);

/* Convert a caller-built tree (same arrays as rq_host_bvh_tree; width 2 ->
 * BVH2 layout, 8 -> CWBVH layout) over the given mesh.  The counterpart of
 * ConvertToGPUBVH2 / ConvertToGPUCompressedWideBVH (src/GPUBVHConverter.h:
 * 13-26), which take a BVHNNode tree from an external builder.  CWBVH leaves
 * must hold 1..3 triangles and nodes at most 8 children in slots 0..n-1. */
rq_status rq_convert_tree(int32_t width, int64_t n_nodes, const int32_t* child_codes,
                          const float* child_boxes, int64_t n_leaves, const int32_t* leaf_first,
                          const int32_t* leaf_count, int64_t n_prim_refs, const int32_t* prim_refs,
                          int32_t root_is_leaf, const float* vertices, int64_t nv,
                          const int32_t* indices, int64_t nt, rq_host_bvh_t* out);

/* Woop transform of one triangle: 3 float4 rows (V0, V1, V2) as
 * WoopifyTriangle emits them (src/GPUBVHConverter.cpp:380-403). */
rq_status rq_woopify(const float v0[3], const float v1[3], const float v2[3], float out_rows[12]);

/* ----------------------------------------------------------- device scenes */
typedef struct rq_scene* rq_scene_t;

/* Register converted buffers as a device-resident scene.  With copy_from_host
 * = 1 the buffers are host pointers and the scene owns device copies; with 0
 * they are device pointers that the caller keeps alive (the reference's
 * rtBind* ownership model, src/TraversalKernelCWBVH.cu:377-385). */
rq_status rq_scene_create(rq_bvh_kind kind, const void* nodes, int64_t node_float4s,
                          const void* woop, int64_t woop_float4s, const int32_t* prim_index,
                          int64_t prim_index_count, int copy_from_host, rq_scene_t* out);
/* Upload a host BVH (from rq_build_bvh) as a device scene. */
rq_status rq_scene_from_host_bvh(rq_host_bvh_t bvh, rq_scene_t* out);
rq_status rq_scene_destroy(rq_scene_t scene);
rq_status rq_scene_device_buffers(rq_scene_t scene, const void** nodes, const void** woop,
                                  const int32_t** prim_index);
/* Buffer lengths of a scene: node and Woop float4s, primitive-map entries. */
rq_status rq_scene_sizes(rq_scene_t scene, int64_t* node_float4s, int64_t* woop_float4s,
                         int64_t* prim_index_count);
int64_t rq_scene_bytes(rq_scene_t scene);

/* ---------------------------------------------------------------- contexts */
/*
 * A context owns the small device scratch of the persistent kernels (the
 * dynamic-fetch ray counter and the error word).  Calls on one context are
 * ordered by the stream they are given; use one context per concurrent stream.
 */
typedef struct rq_ctx* rq_ctx_t;

rq_status rq_ctx_create(rq_ctx_t* out);
rq_status rq_ctx_destroy(rq_ctx_t ctx);
/* Wait for `stream`, read and clear the context's device error word. */
rq_status rq_ctx_check(rq_ctx_t ctx, void* stream);

/* ------------------------------------------------------------------ tracing */
/*
 * Trace `count` rays (device rq_ray[count]) into device rq_hit[count].
 * RQ_CLOSEST follows rtTraceCWBVH / rtTraceBVH2 (src/TraversalKernelCWBVH.cu:387-426,
 * src/TraversalKernelBVH2.cu:190-227): x = t of the closest hit (tmax on a
 * miss), y = Woop address or -1, z/w = u,v of the hit.  RQ_ANY stops a ray at
 * its first accepted triangle; only y != -1 (occluded) is contractual.
 * Ray and hit buffers are float4 records and must be 16-byte aligned (the
 * trace and batch calls refuse others with RQ_ERR_INVALID_ARG).
 * Asynchronous on `stream`; errors detected by the kernel surface at rq_ctx_check.
 */
rq_status rq_trace(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits,
                   int64_t count, rq_query query, const rq_launch* launch, void* stream);

/* Per-ray traversal counters (nodes fetched, triangles tested) written to
 * device int32 arrays, for roofline accounting.  Traverses in the oracle's
 * order (as rq_trace_ordered), so the counts match the CPU restatement's. */
rq_status rq_trace_counted(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits,
                           int64_t count, rq_query query, int32_t* node_visits,
                           int32_t* tri_tests, void* stream);

/* AO bake in one pass (the per-surfel reduction fused into the trace
 * epilogue): any-hit traversal of `count` rays laid out surfel-major (`spp`
 * consecutive rays per surfel, as rq_aorays and GenerateAORaysUniform write
 * them) that adds 1 to occluded[ray / spp] for each occluded ray instead of
 * writing a Hit -- no 16-byte hit store per ray and no separate reduction.
 * `occluded` (device, count / spp entries) accumulates: zero it for a fresh
 * bake.  count must be a multiple of spp.  AO = occluded / spp, equal to
 * rq_ao_reduce over rq_trace any-hit results. */
rq_status rq_trace_ao(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, int64_t count, int spp,
                      uint32_t* occluded, const rq_launch* launch, void* stream);

/* rq_trace with the traversal order of the CPU oracle: no triangle
 * postponing (CWBVH) and no speculative leaf postponing (BVH2).  Its results
 * are bit-identical to the oracle's (t, id, u, v), which is what the parity
 * tests check; rq_trace may differ from it only on exact ties. */
rq_status rq_trace_ordered(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits,
                           int64_t count, rq_query query, void* stream);

/* ------------------------------------------------- several GPUs, one ray set */
/*
 * One ray buffer traced over several devices holding replicas of one scene:
 * the multi-GPU form of rtTraceCWBVH / rtTraceBVH2
 * (src/TraversalKernelCWBVH.cu:387-426, src/TraversalKernelBVH2.cu:190-227).
 * Rays [0, count) split into n_parts contiguous ranges (rq_shard_range: sizes
 * differ by at most one, larger ranges first); range k is traced on
 * devices[k] against scenes[k] (a replica created on that device).  The
 * caller's rays and hits live on devices[0]: range 0 is traced there in
 * place, every other device copies its range in (peer copy into its own
 * staging buffer), traces it and copies its hits back into `hits`.  Devices
 * may repeat.  The trace waits for `stream` (devices[0]) before it starts and
 * returns when every hit is in place, with the first error any part met
 * (kernel errors included, as rq_ctx_check reports them).
 */
typedef struct rq_sharded* rq_sharded_t;
rq_status rq_shard_range(int64_t count, int n_parts, int part, int64_t* begin, int64_t* size);
/* Per part: a context, a stream and (parts 1..) staging buffers for
 * ceil(max_rays / n_parts) rays on that part's device. */
rq_status rq_sharded_create(int n_parts, const int* devices, const rq_scene_t* scenes, int64_t max_rays,
                            rq_sharded_t* out);
rq_status rq_sharded_trace(rq_sharded_t shards, const rq_ray* rays, rq_hit* hits, int64_t count,
                           rq_query query, const rq_launch* launch, void* stream);
rq_status rq_sharded_destroy(rq_sharded_t shards);

/* Defaults used when rq_launch fields are zero (a negative postpone_ratio
 * turns triangle postponing off). */
rq_status rq_default_launch(rq_bvh_kind kind, rq_query query, rq_launch* out);

/* ------------------------------------------------------------ AO ray input */
/*
 * AO rays from a surfel sample cache, one ray per (surfel, sample): surfel
 * s = i / spp, a cosine-weighted hemisphere direction about the surfel normal
 * (concentric disk lifted to the hemisphere), origin = pos + n * radius *
 * offset_scale, tmin/tmax as given.  Follows GenerateAORayUniformKernel
 * (src/ValidationKernels.cu:41-101); the random numbers come from a
 * Philox4x32-10 counter generator keyed by (seed, i) instead of curand XORWOW.
 * pos/nrm are device float4[n_surfels], radius device float[n_surfels].
 */
rq_status rq_aorays(const float* pos, const float* nrm, const float* radius, int64_t n_surfels,
                    int spp, uint64_t seed, float tmin, float tmax, float offset_scale,
                    rq_ray* out_rays, void* stream);

/* Surfels at uniformly chosen triangles (by index) and uniform barycentric
 * points (square-root warp), geometric normals, radius 0.  vertices device
 * float[3*nv], indices device int[3*nt]; outputs device float4/float4/float. */
rq_status rq_sample_surfels(const float* vertices, const int32_t* indices, int64_t nt,
                            int64_t n_surfels, uint64_t seed, float* out_pos, float* out_nrm,
                            float* out_radius, void* stream);

/* Pinhole camera rays, one per pixel centre, row-major (row 0 at the top):
 * eye, look-at point, up vector, vertical field of view in degrees. */
rq_status rq_camera_rays(const float eye[3], const float look[3], const float up[3], float vfov_deg,
                         int width, int height, float tmin, float tmax, rq_ray* out_rays,
                         void* stream);
/* The same rays in tile order, so that a warp's 32 rays cover a compact
 * patch of the image (4 x 8 tiles trace about 6 % faster than rows on a
 * city scene): ray i is pixel (x, y) of tile i / (tile_w * tile_h), tiles
 * row-major across the image, pixels row-major within a tile.  width and
 * height must be multiples of tile_w and tile_h.  Each ray is bit-identical
 * to rq_camera_rays' ray of the same pixel.  No reference counterpart. */
rq_status rq_camera_rays_tiled(const float eye[3], const float look[3], const float up[3], float vfov_deg,
                               int width, int height, int tile_w, int tile_h, float tmin, float tmax,
                               rq_ray* out_rays, void* stream);

/* Surfels at closest-hit points (hit position o + t d, geometric normal from
 * the hit triangle's Woop row V0 -- perpendicular to the triangle -- turned
 * to face the incoming ray, radius 0).  A miss gives a zero normal, for which
 * rq_aorays emits an empty ray (tmin = tmax = 0).  hits must come from a
 * closest-hit trace of this scene; a hit address outside its Woop buffer is
 * treated as a miss. */
rq_status rq_surfels_from_hits(rq_scene_t scene, const rq_ray* rays, const rq_hit* hits,
                               int64_t count, float* out_pos, float* out_nrm, float* out_radius,
                               void* stream);

/* Per-surfel AO fraction (occluded rays / spp) from any-hit results whose rays
 * were generated surfel-major (ray i belongs to surfel i / spp). */
rq_status rq_ao_reduce(const rq_hit* hits, int64_t n_surfels, int spp, float* out_ao,
                       void* stream);

/* ---------------------------------------------------------- Morton sorting */
/* Sort rays by a 32-bit key (10-bit Morton per origin axis inside the given
 * bounds, high bits; direction octant, low bits).  Writes the sorted rays and
 * the permutation (sorted position -> original index). */
rq_status rq_sort_rays(rq_ctx_t ctx, const rq_ray* rays, int64_t count, const float bounds_lo[3],
                       const float bounds_hi[3], rq_ray* sorted_rays, int32_t* perm,
                       void* stream);

/* rq_sort_rays without allocating device memory.  No counterpart in the
 * reference.  Some callers cannot call cudaMalloc -- a plugin inside a host
 * that owns all device memory through its own pool, a service whose
 * device-memory budget was fixed at start-up -- and rq_sort_rays allocates
 * its sort buffers on every call.  This entry point keeps its scratch in one
 * static 20 MiB device array that every GPU loading librq holds until exit,
 * which limits a call to RQ_SORT_STATIC_MAX_RAYS rays (larger counts return
 * RQ_ERR_INVALID_ARG with the limit in rq_last_error).  Outputs are identical
 * to rq_sort_rays's.  Unlike rq_sort_rays, which waits for its stream, the
 * call is stream-ordered and returns with its work queued on `stream`: keep
 * `rays`, `sorted_rays` and `perm` alive until the stream has reached that
 * point.  The first call on a device (with that device current) looks up the
 * array's address; make it before any stream capture.  All calls share the
 * array and leave their contents in it: calls whose work overlaps on the GPU
 * race. */
#define RQ_SORT_STATIC_MAX_RAYS 524288
rq_status rq_sort_rays_static(const rq_ray* rays, int64_t count, const float bounds_lo[3],
                              const float bounds_hi[3], rq_ray* sorted_rays, int32_t* perm,
                              void* stream);

/* -------------------------------------------------------------- batching */
/*
 * A batch traces many (scene, rays, hits) items in one persistent launch over
 * device-resident scenes.  Rays of each item may be Morton-sorted first (items
 * with at least sort_threshold rays); results land at the original ray index.
 * rq_batch_run can be captured into a CUDA graph (use_graph = 1 replays one).
 */
typedef struct rq_batch* rq_batch_t;

typedef struct rq_batch_item {
    rq_scene_t scene;
    const rq_ray* rays;   /* device */
    rq_hit* hits;         /* device */
    int64_t count;
} rq_batch_item;

typedef struct rq_batch_params {
    rq_launch launch;
    int64_t sort_threshold;  /* sort an item's rays when count >= this; <0 never */
    int use_graph;           /* capture the launch sequence in a CUDA graph       */
} rq_batch_params;

rq_status rq_batch_create(rq_ctx_t ctx, const rq_batch_item* items, int n_items, rq_query query,
                          const rq_batch_params* params, rq_batch_t* out);
rq_status rq_batch_run(rq_batch_t batch, void* stream);
/* One stage of rq_batch_run, eagerly (no graph): 1 = Morton sort of the
 * sorted items' rays, 2 = the trace launch alone (reads the rays the last
 * sort left).  Used to time the stages separately. */
rq_status rq_batch_run_stage(rq_batch_t batch, int stage, void* stream);
/* Kernels one rq_batch_run launches (counted from its captured graph when
 * use_graph is set, else from the stages it runs). */
int rq_batch_kernel_count(rq_batch_t batch);
int64_t rq_batch_total_rays(rq_batch_t batch);
rq_status rq_batch_destroy(rq_batch_t batch);

/* ---------------------------------------------------------------- autotune */
/*
 * Time the candidate launch shapes (block size, shared-memory stack depth,
 * postponing on/off) on the given rays, then, on the fastest shape, the
 * dynamic-fetch refill thresholds (fetch_nd, fetch_nw) and the postponing
 * ratio, and return the fastest.  When cache_path is non-null the choice is
 * stored there keyed by device, BVH kind, query and size class, and later
 * calls read it back.
 */
rq_status rq_autotune(rq_ctx_t ctx, rq_scene_t scene, const rq_ray* rays, rq_hit* hits,
                      int64_t count, rq_query query, const char* cache_path, rq_launch* out,
                      void* stream);

/* Tune a whole batch: sort threshold (never / large items / all) x block size
 * x shared-memory stack depth, then refill thresholds and postponing ratio on
 * the fastest of those, timed on the batch itself, cached like rq_autotune.
 * use_graph is set when `stream` is not the default stream. */
rq_status rq_autotune_batch(rq_ctx_t ctx, const rq_batch_item* items, int n_items, rq_query query,
                            const char* cache_path, rq_batch_params* out, void* stream);

/* ----------------------------------------------------------------- serving */
/*
 * A continuous-batching AO bake server.  The HBM budget is one device pool
 * allocated at creation; every request buffer lives in it.  Requests are cut
 * into pieces of at most max_batch_rays rays (whole surfels for bake
 * requests) that each fit the pool, so a request larger than one launch is
 * split rather than refused.  Pieces are admitted in arrival order while the
 * pool can give them their buffers (admission by bytes: the bytes in use
 * never exceed the budget, and queued pieces wait for running ones to give
 * theirs back), gathered into persistent batch launches on several streams
 * (so batches overlap on the device), and completed by copying results back
 * to the caller's host buffer; a request completes with its last piece.
 */
typedef struct rq_server* rq_server_t;

typedef struct rq_server_params {
    int64_t hbm_budget_bytes;   /* device pool for request buffers (48 B per ray of a ray request) */
    int64_t max_batch_rays;     /* rays per launch and per piece (0 = budget / (48 x streams))      */
    int streams;                /* concurrent batch streams (default 3)          */
    rq_query query;
    rq_launch launch;
} rq_server_params;

typedef struct rq_request_stats {
    double submit_ms;     /* host monotonic clock, ms                           */
    double start_ms;      /* when its first piece was launched                  */
    double done_ms;       /* when its last results were back in the caller's buffer */
    int64_t rays;
    int32_t batch_id;     /* launch of its first piece                          */
    int32_t status;       /* rq_status of the request                           */
} rq_request_stats;

/* Pool accounting of a server (no reference counterpart). */
typedef struct rq_server_memory_stats {
    int64_t pool_bytes;         /* the HBM budget (rounded down to 256 B)           */
    int64_t in_use_bytes;       /* held by admitted pieces now                      */
    int64_t peak_in_use_bytes;  /* most ever held at once (<= pool_bytes)           */
    int64_t admission_waits;    /* times the oldest queued piece waited for bytes   */
    int64_t pieces;             /* pieces queued so far                             */
    int64_t max_batch_rays;     /* rays per launch and per piece in effect          */
} rq_server_memory_stats;

rq_status rq_server_create(const rq_server_params* params, rq_server_t* out);
rq_status rq_server_add_scene(rq_server_t server, rq_scene_t scene, int32_t* scene_id);
/* host_rays must stay valid and host_hits writable until the request completes.
 * Pinned host memory gives overlapped copies; pageable memory works too. */
rq_status rq_server_submit(rq_server_t server, int32_t scene_id, const rq_ray* host_rays,
                           rq_hit* host_hits, int64_t count, uint64_t* ticket);
/* timeout_ms < 0 waits without limit. */
/* An AO bake request: n_surfels host surfels (pos, nrm float4 each, radius
 * float each or NULL for 0) and `spp` rays per surfel generated on the device
 * exactly as rq_aorays does (seed, tmin, tmax, offset_scale), traced any-hit
 * with the occluded rays counted per surfel in the trace epilogue; host_ao
 * (n_surfels floats) receives occluded / spp, equal to rq_aorays + rq_trace
 * + rq_ao_reduce.  Only the surfels (36 B each) go to the device and 4 B per
 * surfel come back.  A piece occupies 36 B per surfel + 4 B per surfel +
 * 32 B per ray of the pool (rounded to 256 B per buffer); RQ_ERR_BUDGET if
 * one surfel's rays exceed max_batch_rays or its buffers the pool,
 * RQ_ERR_INVALID_ARG on a closest-hit server. */
rq_status rq_server_submit_bake(rq_server_t server, int32_t scene_id, const float* host_pos,
                                const float* host_nrm, const float* host_radius, int64_t n_surfels,
                                int spp, uint64_t seed, float tmin, float tmax, float offset_scale,
                                float* host_ao, uint64_t* ticket);
rq_status rq_server_wait(rq_server_t server, uint64_t ticket, int64_t timeout_ms,
                         rq_request_stats* stats);
/* Cancels a request none of whose pieces has started (RQ_ERR_NOT_FOUND
 * otherwise); its wait returns RQ_ERR_CANCELLED. */
rq_status rq_server_cancel(rq_server_t server, uint64_t ticket);
rq_status rq_server_memory(rq_server_t server, rq_server_memory_stats* out);
rq_status rq_server_destroy(rq_server_t server);

/* ------------------------------------------------- procedural test scenes */
/*
 * Seeded synthetic meshes standing in for the reference's missing mesh.dat.
 * The library allocates *vertices (3*nv floats) and *indices (3*nt ints);
 * release them with rq_free_mesh.
 *   heightfield_boxes: (grid+1)^2-vertex heightfield over [0,1]^2, heights
 *     U[0,1], plus n_boxes axis-aligned boxes (12 triangles each), centres
 *     U over [0,1]^3, edges U[box_min, box_max].
 *   city: n_buildings boxes/prisms on a grid with log-normal heights over a
 *     ground plane.
 *   spheres_terrain: displaced subdivided spheres over displaced terrain tiles.
 */
rq_status rq_gen_heightfield_boxes(uint64_t seed, int grid, int n_boxes, float box_min,
                                   float box_max, float** vertices, int64_t* nv,
                                   int32_t** indices, int64_t* nt);
rq_status rq_gen_city(uint64_t seed, int n_buildings, float** vertices, int64_t* nv,
                      int32_t** indices, int64_t* nt);
rq_status rq_gen_spheres_terrain(uint64_t seed, int64_t target_tris, float** vertices,
                                 int64_t* nv, int32_t** indices, int64_t* nt);
void rq_free_mesh(float* vertices, int32_t* indices);

/* ------------------------------------------------------ scene / sample files */
/*
 * The reference's input files (src/main.cpp:31-45, :52-64), little-endian:
 *   mesh.dat        int32 nV, int32 nT, float3 v[nV], int3 tri[nT], int32 material[nT]
 *   samplecache.dat int32 SX, int32 SY, float4 pos[SX*SY], float4 nrm[SX*SY],
 *                   float radius[SX*SY]
 * Loaders check every count against the file length and every index against
 * nV (RQ_ERR_INVALID_ARG otherwise; RQ_ERR_NOT_FOUND if the file cannot be
 * opened) and return malloc'd arrays: release the mesh's with rq_free_mesh,
 * materials and sample arrays with rq_free_host.  `materials` may be NULL
 * (not returned / written as zeros).
 */
rq_status rq_load_mesh_dat(const char* path, float** vertices, int64_t* nv, int32_t** indices,
                           int64_t* nt, int32_t** materials);
rq_status rq_save_mesh_dat(const char* path, const float* vertices, int64_t nv,
                           const int32_t* indices, int64_t nt, const int32_t* materials);
rq_status rq_load_samplecache_dat(const char* path, int32_t* size_x, int32_t* size_y, float** pos,
                                  float** nrm, float** radius);
rq_status rq_save_samplecache_dat(const char* path, int32_t size_x, int32_t size_y,
                                  const float* pos, const float* nrm, const float* radius);
void rq_free_host(void* p);

/* Converted-scene files (this library's format "RQSCENE1": header with kind,
 * counts, bounds and an FNV-1a checksum, then the node, Woop and
 * primitive-map buffers), so a scene reloads without a rebuild.  A loaded
 * handle has buffers only: rq_host_bvh_tree returns RQ_ERR_NOT_FOUND.
 * A malformed or corrupt file gives RQ_ERR_BAD_SCENE. */
rq_status rq_host_bvh_save(rq_host_bvh_t bvh, const char* path);
rq_status rq_host_bvh_load(const char* path, rq_host_bvh_t* out);

/* ----------------------------------------------- reference-shaped adapters */
/*
 * Same names, argument meaning and byte layouts as the reference's host entry
 * points, so a caller written against them links unchanged (float4/Ray/Hit
 * are passed as void* here; librq also exports C++-linkage overloads with the
 * exact reference signatures).  One global bound scene per BVH kind, as in the
 * reference; tracing is synchronous on the legacy default stream and returns
 * the kernel's error status instead of aborting.
 *   rtBindCWBVHData  src/TraversalKernelCWBVH.h:3-6 (src/TraversalKernelCWBVH.cu:377-385)
 *   rtTraceCWBVH     src/TraversalKernelCWBVH.h:8-11 (src/TraversalKernelCWBVH.cu:387-426)
 *   rtBindBVH2Data   src/TraversalKernelBVH2.h:3-6 (src/TraversalKernelBVH2.cu:180-188)
 *   rtTraceBVH2      src/TraversalKernelBVH2.h:8-11 (src/TraversalKernelBVH2.cu:190-227)
 *   GenerateAORaysUniform src/ValidationKernels.h:3-9 (src/ValidationKernels.cu:140-187):
 *     host surfel arrays in, a new device Ray buffer out (caller frees it with
 *     cudaFree), tmin 0.01, tmax 1e20, origin offset radius/2.
 */
rq_status rq_rtBindCWBVHData(const void* nodes, const void* woop, const int32_t* prim_index);
rq_status rq_rtTraceCWBVH(void* rays, void* hits, int ray_count);
rq_status rq_rtBindBVH2Data(const void* nodes, const void* woop, const int32_t* prim_index);
rq_status rq_rtTraceBVH2(void* rays, void* hits, int ray_count);
void* rq_GenerateAORaysUniform(int num_texels, int rays_per_texel, const float* pos,
                               const float* nrm, const float* radius);
/* Any-hit twins of rtTrace* (the reference has only closest-hit). */
rq_status rq_rtOccludedCWBVH(void* rays, void* hits, int ray_count);
rq_status rq_rtOccludedBVH2(void* rays, void* hits, int ray_count);

/* Synchronous device-to-device copy, and cudaFree of a buffer this library
 * returned (rq_GenerateAORaysUniform). */
rq_status rq_device_copy(void* dst, const void* src, int64_t bytes);
rq_status rq_device_free(void* p);

/* ------------------------------------------------------------ GPU build */
/*
 * A CWBVH scene built on the device from device-resident vertices (3*nv
 * floats) and indices (3*nt ints) on `stream`.  The binary tree comes from
 * the triangles in Morton order, either as Karras's radix tree
 * (RQ_GPU_BUILD_LBVH: fastest) or by parallel locally-ordered clustering
 * (RQ_GPU_BUILD_PLOC: merged boxes of least area; better trees).  With
 * `split_budget` > 0 (percent of nt, at most 400; 0 = none) triangles whose
 * boxes are much larger than they are are first cut into references along
 * a grid's planes (Karras and Aila 2013), at most nt * split_budget / 100
 * extra, and a triangle may then be stored more than once.  Then
 * `optimize_passes` bottom-up passes of treelet restructuring (7-leaf
 * treelets rebuilt SAH-optimally, a warp per treelet; 0 = none), then a
 * top-down collapse to
 * 8-wide nodes written in the CWBVH format with Woop rows and the primitive
 * map.  Much faster to build than rq_build_bvh, slower to trace; the scene
 * owns its buffers (rq_scene_destroy).  No reference counterpart (the
 * reference builds on the host with Embree).  Indices outside [0, nv) give
 * RQ_ERR_INVALID_ARG, as do an unknown method and a budget outside
 * [0, 400].  Synchronises `stream` once per tree level (and once per
 * clustering round).
 */
#define RQ_GPU_BUILD_LBVH 0
#define RQ_GPU_BUILD_PLOC 1
/* OR-ed into `method`: restructure each treelet with one thread instead of
 * one warp (slower; the same trees, byte for byte). */
#define RQ_GPU_BUILD_THREAD_TREELETS 0x100
rq_status rq_build_scene_gpu(const float* vertices, int64_t nv, const int32_t* indices, int64_t nt, int method,
                             int optimize_passes, int split_budget, rq_scene_t* out, void* stream);

/* ------------------------------------------------------- instancing (TLAS) */
/*
 * Two-level scenes (no reference counterpart: the reference traces one flat
 * scene).  A top-level CWBVH is built over instances of bottom-level CWBVH
 * scenes; instance k places scene blas[blas_index[k]] with the affine
 * object-to-world transform object_to_world[12 k .. 12 k + 11] (3 x 4,
 * row-major: world = M [p; 1]).  Rays are traced in world space; each hit
 * reports t (the same in world and object space), the Woop address within
 * its bottom-level scene, u, v, and -- in instance_out, if not NULL -- the
 * instance (-1 on a miss).  The bottom-level scenes are borrowed: keep them
 * alive while the top level is in use.  Singular or non-finite transforms,
 * BVH2 scenes and out-of-range indices give RQ_ERR_INVALID_ARG.
 */
typedef struct rq_tlas* rq_tlas_t;
rq_status rq_tlas_create(const rq_scene_t* blas, int n_blas, const float* object_to_world,
                         const int32_t* blas_index, int64_t n_instances, rq_tlas_t* out);
rq_status rq_tlas_destroy(rq_tlas_t tlas);
/* The top-level tree alone, built on the host from the bottom-level scenes'
 * bounds (6 floats each: lo xyz, hi xyz): nodes, instance rows in place of
 * Woop rows and the (instance, bottom-level index, -1) map, as a host BVH
 * handle (rq_host_bvh_buffers / rq_host_bvh_free).  rq_tlas_create runs this
 * with the scenes' bounds and uploads the result. */
rq_status rq_tlas_build_host(const float* blas_bounds, int n_blas, const float* object_to_world,
                             const int32_t* blas_index, int64_t n_instances, rq_host_bvh_t* out);
/* Host copies of the top-level buffers: nodes, instance rows (the
 * world-to-object transform, 3 float4 per instance slot) and the map
 * (instance, bottom-level index, -1) per row. */
rq_status rq_tlas_buffers(rq_tlas_t tlas, const float** nodes, int64_t* node_float4s,
                          const float** rows, int64_t* row_float4s, const int32_t** map);
/* launch: NULL for the defaults; only postpone_ratio (triangle / instance
 * postponing as in rq_trace, but off unless a positive ratio is given: off is
 * the oracle's traversal order), fetch_nd / fetch_nw and step_limit are used. */
rq_status rq_trace_instanced(rq_ctx_t ctx, rq_tlas_t tlas, const rq_ray* rays, rq_hit* hits,
                             int32_t* instance_out, int64_t count, rq_query query,
                             const rq_launch* launch, void* stream);

/* ------------------------------------------------------------- device info */
int rq_device_sm_count(void);
/* L2 read-bandwidth probe (a measurement utility; no reference counterpart):
 * every thread of a grid of SMs x 8 blocks x 256 threads reads `buf`
 * (device, `bytes` a multiple of 16, 16-byte aligned) `reps` times with
 * coalesced L1-bypassing 16-byte loads (a warp's load covers 512 contiguous
 * bytes), four in flight per thread, and folds the words into `sink` (device,
 * 4 bytes) only if they XOR to a magic value, so the loads stay live.  A
 * buffer well inside L2 gives the L2 read bandwidth: time the call with
 * events on `stream` and divide bytes * reps by the time. */
rq_status rq_probe_l2_read(const void* buf, int64_t bytes, int reps, uint32_t* sink, void* stream);
/* The same probe with its launch shape given: SMs x blocks_per_sm blocks
 * (1..64) and `loads` (4 or 8) loads in flight per thread. */
rq_status rq_probe_l2_read_shape(const void* buf, int64_t bytes, int reps, int blocks_per_sm, int loads,
                                 uint32_t* sink, void* stream);
/* Library build identification: "rq <version> sm_100a". */
const char* rq_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RQ_H */
