/*
 * rq.h — C ABI of the B200 ray-query engine (librq.so).
 *
 * This is the drop-in boundary for the reference's BVH build and software
 * traversal path.  Every entry point names the reference interface it stands
 * in for (file:line inside the reference project).  Conventions:
 *   - plain C types only; device buffers are passed as raw device pointers,
 *     CUDA streams as opaque `rq_stream` (a cudaStream_t, NULL = legacy stream);
 *   - every call returns an rq_status; no C++ exception crosses the ABI;
 *   - calls are stream-ordered and asynchronous unless documented otherwise;
 *   - one rq_ctx owns its scratch memory, so calls that share a ctx must be
 *     ordered on one stream (use one ctx per concurrently used stream).
 */
#ifndef RQ_H
#define RQ_H

#include "rq_layouts.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void* rq_stream;
typedef struct rq_ctx rq_ctx;
typedef struct rq_bvh rq_bvh;

typedef enum rq_status {
    RQ_OK = 0,
    RQ_ERR_INVALID_ARG = 1,     /* null pointer, zero size where one is needed, bad flag */
    RQ_ERR_SIZE = 2,            /* an output buffer is smaller than required */
    RQ_ERR_CUDA = 3,            /* a CUDA runtime call failed (rq_ctx_last_error has text) */
    RQ_ERR_OOM = 4,             /* device allocation failed */
    RQ_ERR_DEVICE_TIMEOUT = 5,  /* a bounded device-side wait gave up */
    RQ_ERR_UNSUPPORTED = 6,     /* input outside what the kernels handle (e.g. > 2^27 triangles) */
    RQ_ERR_BUDGET = 7,          /* serving: request does not fit the memory budget */
    RQ_ERR_NO_DEVICE = 8,       /* no CUDA device, or the device is not sm_100 */
    RQ_ERR_STATE = 9,           /* handle used before it was built */
    RQ_ERR_CANCELLED = 10       /* serving: the request was cancelled before it was admitted */
} rq_status;

/* ------------------------------------------------------------------ */
/* Context                                                             */
/* ------------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  Fails with RQ_ERR_NO_DEVICE on
 * anything other than a compute-capability 10.x device. */
int rq_ctx_create(int device, rq_ctx** out);
int rq_ctx_destroy(rq_ctx* ctx);
const char* rq_status_string(int status);
/* Text of the last error recorded on this context ("" if none). */
const char* rq_ctx_last_error(const rq_ctx* ctx);
/* Synchronise `stream`, then read and clear the context's device error word
 * (set by kernels whose bounded waits gave up).  RQ_OK when clean. */
int rq_ctx_check(rq_ctx* ctx, rq_stream stream);
/* Bytes of device scratch the context currently holds. */
uint64_t rq_ctx_scratch_bytes(const rq_ctx* ctx);
/* Check of the failure path of bounded device waits: one thread waits for
 * the device word *flag to leave 0, with the wait the grid barriers use,
 * for at most `limit` polls (<= 2^20, 64 ns apart).  If nothing changes the
 * word, the wait gives up and the next rq_ctx_check reports
 * RQ_ERR_DEVICE_TIMEOUT; the context stays usable. */
int rq_debug_wait_timeout(rq_ctx* ctx, const uint32_t* flag, uint32_t limit, rq_stream stream);

/* Launch shape of the context's persistent shadow/AO traversal
 * (rq_render_shadow_ao).  Results do not depend on it. */
typedef struct rq_trace_tuning {
    uint32_t threads;  /* per block: 64, 128 or 256 (default 128) */
    uint32_t chunk;    /* ray ids a warp takes per refill: 32 or 64 (default 32) */
    uint32_t reg_cap;  /* registers per thread the launch bounds allow: 0 (no bound), 64, 72 (threads
                          64 or 128 only) or 80 (default) */
    uint32_t top_levels; /* 0, or 4: each block stages the tree's top 4 levels (<= 85 nodes) in shared memory */
    uint32_t speculative; /* 1: lanes holding a leaf keep taking inner nodes while the warp searches
                             (the frame only reports hit or miss, so the order does not show) */
    uint32_t refill_min;  /* a warp hands new rays to its idle lanes only once at least this many of
                             its 32 lanes are idle (or all are): 1..32; 0 means 1 */
    uint32_t leaf_batch;  /* 0: rays finish and lanes refill between rounds only.  1..32: a lane whose
                             ray runs out of nodes reports at once and idle lanes refill inside the
                             node loop, which hands over to the leaf tests once this many lanes hold a
                             leaf (speculative shapes only) */
} rq_trace_tuning;
int rq_ctx_trace_tuning_get(const rq_ctx* ctx, rq_trace_tuning* out);
/* RQ_ERR_INVALID_ARG for a shape that has no kernel. */
int rq_ctx_trace_tuning_set(rq_ctx* ctx, const rq_trace_tuning* t);

/* Schedule of the context's camera traversal (rq_render_gbuffer).  Results
 * do not depend on it. */
typedef struct rq_camera_tuning {
    uint32_t engine;      /* 0: one ray per thread, 8x4-pixel tiles per warp (default); 1: the
                             persistent refilling engine with in-loop refill (128-thread blocks,
                             64 registers) */
    uint32_t refill_min;  /* engine: idle lanes before a refill, 1..32 (0 means 1) */
    uint32_t leaf_batch;  /* engine: parked leaves that end the node loop, 1..32 (0 means 32) */
} rq_camera_tuning;
int rq_ctx_camera_tuning_get(const rq_ctx* ctx, rq_camera_tuning* out);
int rq_ctx_camera_tuning_set(rq_ctx* ctx, const rq_camera_tuning* t);

/* ------------------------------------------------------------------ */
/* Mesh generation and deformation (inputs of the BVH path)            */
/* ------------------------------------------------------------------ */

/* Height-field grid on the host: (qx+1)*(qy+1) vertices on [x0,x1]x[y0,y1],
 * z = amp*sin(freq*x)*cos(freq*y) + N(0, sigma) per vertex (seeded), two
 * triangles per quad wound like generate_dynamic_grid_mesh
 * (include/radv_bvh.hpp:257-274).  `pos` gets 3 floats per vertex, `idx`
 * 6 uint32 per quad.  Host pointers.  Replaces the input side of
 * MeshGenerator::createTessellatedTerrain (common/mesh_gen.hpp:29-83). */
int rq_scene_grid(uint32_t qx, uint32_t qy, float x0, float x1, float y0, float y1,
                  float amp, float freq, float sigma, uint64_t seed,
                  float* pos, uint32_t* idx);

/* Rays on the host for the plain workload: origins uniform in
 * [x0,x1]x[y0,y1] at height z, directions normalize(U(-s,s), U(-s,s), -1),
 * the given tmin/tmax; SplitMix64 (seeded), double precision rounded once.
 * Host pointer `rays` (n entries). */
int rq_scene_rays_down(uint32_t n, float x0, float x1, float y0, float y1, float z, float spread, float tmin,
                       float tmax, uint64_t seed, rq_ray* rays);

/* Device kernel: out[v].z = base[v].z + amp*sin(t + freq*base[v].x), x and y
 * copied.  3 floats per vertex, device pointers (in-place allowed).  The
 * per-frame deformation step (benchmarks/expA_async/shaders/mesh_deform.comp:25-34). */
int rq_deform_wave(rq_ctx* ctx, const float* base, float* out, uint32_t num_vertices,
                   float t, float amp, float freq, rq_stream stream);
/* The same with the time in device memory: `state` (device, 2 uint32) holds
 * t as float bits and a zeroed work word; after the launch t has advanced
 * by dt.  A recorded sequence of frames then animates without host input. */
int rq_deform_wave_step(rq_ctx* ctx, const float* base, float* out, uint32_t num_vertices,
                        uint32_t* state, float dt, float amp, float freq, rq_stream stream);

/* ------------------------------------------------------------------ */
/* BVH build (LBVH: Morton codes, onesweep radix sort, Karras emission, */
/* atomic bottom-up refit, BVH4 collapse)                              */
/* ------------------------------------------------------------------ */

#define RQ_BUILD_BVH4 1u /* also collapse to the 4-wide layout (needed by rq_trace) */
/* Split like SoftwareBVH::recursiveBuild (common/software_bvh.hpp:90-175) instead
 * of Morton order: median of the longest centroid axis, leaves of <= max_leaf
 * primitives or of centroids spanning < 1e-6.  Where no centroid value
 * repeats inside a node on its split axis, the binary nodes (boxes, child
 * links, leaf offsets and counts) equal the reference's; the order of the
 * triangles inside a leaf is the x-centroid order (the reference's is
 * nth_element's).  Slower than the LBVH (one round per tree level); the
 * sorted Morton keys of the handle are not written. */
#define RQ_BUILD_MEDIAN 2u
/* The LBVH's Karras hierarchy above every node of at most RQ_SAH_SUBTREE_MAX
 * triangles; each such subtree (a contiguous range of the Morton order) is
 * rebuilt top down by binned SAH (16 bins per axis over the node's centroid
 * bounds for nodes of more than 32 triangles, 8 for smaller nodes; the
 * smallest float(nL)*SA(left) + float(nR)*SA(right), first by
 * axis then by bin on ties, a stable partition, leaves of at most max_leaf
 * triangles; the middle of the range where no axis has a centroid extent or
 * 24 levels are reached).  Fewer node visits per ray than the plain LBVH
 * (about 23 % on the 1080p frame's shadow rays; a binned SAH over the whole
 * mesh: 25 %); Morton keys and the sort are the LBVH's, the
 * permutation differs inside the rebuilt subtrees.  Not with
 * RQ_BUILD_MEDIAN. */
#define RQ_BUILD_SAH 4u
#define RQ_SAH_SUBTREE_MAX 16384u

/* Build a binary BVH over `num_triangles` triangles.  Device pointers.
 * `positions`: float xyz per vertex with `stride_bytes` between vertices
 * (>= 12, multiple of 4).  `indices`: 3 uint32 per triangle, or NULL for a
 * non-indexed mesh (triangle i uses vertices 3i, 3i+1, 3i+2).
 * Leaves hold at most `max_leaf` (1..16) primitives.  The result, in the
 * byte layouts of common/software_bvh.hpp, lives in a library-owned handle.
 * If *out is non-NULL and has capacity for num_triangles, it is rebuilt in
 * place (the per-frame path; no allocation).
 * Replaces SoftwareBVH::build (common/software_bvh.hpp:35-87); with
 * RQ_BUILD_BVH4 also SoftwareBVH4::fromBVH2 (:193-199). */
int rq_build(rq_ctx* ctx, const float* positions, uint32_t stride_bytes, uint32_t num_vertices,
             const uint32_t* indices, uint32_t num_triangles, uint32_t max_leaf, uint32_t flags,
             rq_bvh** out, rq_stream stream);

/* Collapse the handle's binary BVH to the 4-wide layout with the greedy
 * largest-surface-area rule of SoftwareBVH4::collapse
 * (common/software_bvh.hpp:202-291), nodes in the same depth-first order. */
int rq_collapse4(rq_ctx* ctx, rq_bvh* bvh, rq_stream stream);

/* Refit after the vertices moved: same topology, new triangle copies and
 * boxes for both layouts.  `positions` as in rq_build; the index buffer must
 * be the one the handle was built with (it is not stored).  Replaces the
 * driver refit (common/vk_bvh.cpp:558-611) for this BVH. */
int rq_refit(rq_ctx* ctx, rq_bvh* bvh, const float* positions, uint32_t stride_bytes,
             const uint32_t* indices, rq_stream stream);

/* Wrap foreign device arrays (for example a SoftwareBVH uploaded from the
 * host) in a handle: the arrays are copied.  `perm` maps leaf order to
 * original primitive IDs and may be NULL (then IDs are leaf-order indices,
 * as the reference shaders report them). */
int rq_bvh_import2(rq_ctx* ctx, const rq_bvh2_node* nodes, uint32_t num_nodes,
                   const rq_triangle* tris, const uint32_t* perm, uint32_t num_triangles,
                   rq_bvh** out, rq_stream stream);
int rq_bvh_import4(rq_ctx* ctx, const rq_bvh4_node* nodes, uint32_t num_nodes,
                   const rq_triangle* tris, const uint32_t* perm, uint32_t num_triangles,
                   rq_bvh** out, rq_stream stream);

typedef struct rq_bvh_info {
    uint32_t num_triangles;
    uint32_t num_nodes2;   /* binary nodes (0 if the handle only has a 4-wide BVH) */
    uint32_t num_nodes4;   /* 4-wide nodes (0 until collapsed) */
    uint32_t depth4;       /* levels of the 4-wide tree (root = 1) */
    uint32_t max_leaf;
    uint32_t stack_bound;  /* traversal stack entries the tree can need */
    uint64_t device_bytes; /* bytes the handle holds on the device */
} rq_bvh_info;

/* Synchronises the handle's last build stream, then fills `info`. */
int rq_bvh_info_get(rq_bvh* bvh, rq_bvh_info* info);

/* Copy the layouts out (device-to-device or device-to-host; `host` selects
 * which the destination pointers are).  Any destination may be NULL.
 * Capacities are in elements; RQ_ERR_SIZE when one is too small.
 * morton/sorted_ids expose the sort stage (keys and permutation). */
int rq_bvh_download(rq_bvh* bvh, int host,
                    rq_bvh2_node* nodes2, uint32_t cap_nodes2,
                    rq_triangle* tris, uint32_t cap_tris,
                    rq_bvh4_node* nodes4, uint32_t cap_nodes4,
                    uint32_t* perm, uint32_t cap_perm);
int rq_bvh_download_sort(rq_bvh* bvh, int host, uint32_t* morton, uint32_t* sorted_ids, uint32_t cap);
int rq_bvh_destroy(rq_bvh* bvh);

/* ------------------------------------------------------------------ */
/* Traversal                                                           */
/* ------------------------------------------------------------------ */

/* flags */
#define RQ_TRACE_CLOSEST 0u     /* full traversal, nearest hit (gl_RayFlagsNoneEXT/Opaque) */
#define RQ_TRACE_ANY 1u         /* stop at the first accepted hit (TerminateOnFirstHit) */
#define RQ_TRI_WATERTIGHT 0u    /* Woop-Benthin-Wald 2013 watertight test */
#define RQ_TRI_MT 2u            /* Moller-Trumbore with the reference's arithmetic */

/* Trace `n` rays against the handle's 4-wide BVH.  Accept tmin <= t < best,
 * best starting at the ray's tmax.  Hits carry the ORIGINAL primitive ID.
 * `bary` (2 floats per ray, barycentrics of v1 and v2) and `stats`
 * (per-ray node/triangle test counts) may be NULL.
 * Stands in for rayQueryEXT over a BLAS (benchmarks/exp0_probe/shaders/
 * probe_triangle.comp:28-64) and the software traversals of
 * software_bvh_bvh4.comp:60-196. */
int rq_trace(rq_ctx* ctx, const rq_bvh* bvh, const rq_ray* rays, uint32_t n, uint32_t flags,
             rq_hit* hits, float* bary, rq_ray_stats* stats, rq_stream stream);

/* The reference's own software traversal semantics, kept for parity and for
 * callers that depend on its quirks:
 *  - rq_trace_ref_bvh4: software_bvh_bvh4.comp:96-195 (24-entry stack that
 *    drops overflow, leaves tested inline far-to-near, MT with |a|<1e-7,
 *    1/d replaced by 1e6 when |d|<=1e-6).  Writes RayStats and hits; hit IDs
 *    are leaf-order indices as the shader reports them.
 *  - rq_trace_ref_bvh2: software_bvh_lds.comp:86-175 (32-entry stack, MT with
 *    |a|<1e-8, accept t>t_eps) — t_eps 0.001 for the LDS shader, 0.01 for
 *    software_bvh_procedural.comp.  Writes the hitFound flag per ray. */
int rq_trace_ref_bvh4(rq_ctx* ctx, const rq_bvh4_node* nodes, const rq_triangle* tris,
                      const rq_ray* rays, uint32_t n, rq_ray_stats* stats, rq_hit* hits,
                      rq_stream stream);
int rq_trace_ref_bvh2(rq_ctx* ctx, const rq_bvh2_node* nodes, const rq_triangle* tris,
                      const rq_ray* rays, uint32_t n, float t_eps, uint32_t* hit_flags,
                      rq_stream stream);

/* Procedural rays of software_bvh_bvh4.comp:60-94: coherent = 1024-wide
 * camera grid from cam_pos toward look_at (x0.55 field), otherwise PCG-hashed
 * origins in [-40,40]x[15,30]x[-40,40] heading down.  tmin 0.01, tmax 1000. */
int rq_gen_rays_procedural(rq_ctx* ctx, const float cam_pos[3], const float look_at[3],
                           uint32_t count, uint32_t coherent, rq_ray* rays, rq_stream stream);

/* ------------------------------------------------------------------ */
/* Batches: many meshes built in one launch and traced in one launch   */
/* ------------------------------------------------------------------ */

typedef struct rq_batch rq_batch;

/* One mesh of a batch inside shared vertex and index buffers: its vertices
 * start at vertex_offset, its triangles (3 mesh-local uint32 indices each) at
 * triangle_offset.  At most 2^20 triangles per mesh. */
typedef struct rq_mesh_desc {
    uint32_t vertex_offset;
    uint32_t num_vertices;
    uint32_t triangle_offset;
    uint32_t num_triangles;
} rq_mesh_desc;

/* Allocate a batch for the given meshes (host array; copied).  Triangle
 * ranges must not overlap.  The batch owns its arrays and build scratch. */
int rq_batch_create(rq_ctx* ctx, const rq_mesh_desc* meshes, uint32_t num_meshes, uint32_t max_leaf,
                    rq_batch** out);
/* Build every mesh's binary and 4-wide BVH in ONE persistent launch: each
 * thread block builds one mesh at a time (largest first) with the same steps
 * as rq_build, so each mesh's bytes equal a separate rq_build of it.  Device
 * pointers; stride as in rq_build.  The first build synchronises once to
 * read the depths; later builds stay asynchronous. */
int rq_batch_build(rq_ctx* ctx, rq_batch* batch, const float* positions, uint32_t stride_bytes,
                   const uint32_t* indices, rq_stream stream);
/* Trace rays of any meshes of the batch in ONE persistent launch.  ray_mesh[i]
 * names ray i's mesh; ray_flags[i] (may be NULL: `flags` for all) selects any
 * hit (RQ_TRACE_ANY) per ray; RQ_TRI_MT in `flags` selects the triangle
 * test.  Primitive IDs are mesh-local original triangle ids.  stats may be NULL. */
int rq_batch_trace(rq_ctx* ctx, const rq_batch* batch, const rq_ray* rays, const uint32_t* ray_mesh,
                   const uint32_t* ray_flags, uint32_t n, uint32_t flags, rq_hit* hits, rq_ray_stats* stats,
                   rq_stream stream);
/* Per-mesh counts (synchronises) and downloads, as rq_bvh_info_get /
 * rq_bvh_download for one mesh of the batch. */
int rq_batch_info_get(rq_batch* batch, uint32_t mesh, rq_bvh_info* info);
int rq_batch_download(rq_batch* batch, uint32_t mesh, int host, rq_bvh2_node* nodes2, uint32_t cap_nodes2,
                      rq_triangle* tris, uint32_t cap_tris, rq_bvh4_node* nodes4, uint32_t cap_nodes4,
                      uint32_t* perm, uint32_t cap_perm);
int rq_batch_destroy(rq_batch* batch);

/* ------------------------------------------------------------------ */
/* Two-level scenes: instances of BLAS handles under a top-level BVH   */
/* ------------------------------------------------------------------ */

typedef struct rq_tlas rq_tlas;

/* One instance, as VkAccelerationStructureInstanceKHR describes it
 * (benchmarks/exp1_visbuf/visbuf_main.cpp:762-771). */
typedef struct rq_instance {
    float transform[12];  /* object -> world, row-major 3x4 (VkTransformMatrixKHR) */
    uint32_t instance_id; /* reported as rq_hit.instance_id (instanceCustomIndex) */
    uint32_t mask;        /* seen by rays whose cull mask shares a bit with it */
    const rq_bvh* blas;   /* built with RQ_BUILD_BVH4; many instances may share one */
} rq_instance;

/* Build the top level over `num_instances` instances (host array; copied).
 * The handle refers to the BLAS arrays: keep them alive and unchanged (an
 * in-place rebuild or refit of a BLAS needs a new rq_tlas_build).  Replaces
 * the driver TLAS build of common/vk_bvh.cpp:237-336.  Synchronises once. */
int rq_tlas_build(rq_ctx* ctx, const rq_instance* instances, uint32_t num_instances, rq_tlas** out,
                  rq_stream stream);
/* Trace rays through the scene: hits carry the instance id and the BLAS's
 * mesh-local primitive id; t is world-space.  `cull_mask` as rayQueryEXT's
 * cullMask (0xff: every instance).  Flags as rq_trace. */
int rq_tlas_trace(rq_ctx* ctx, const rq_tlas* tlas, const rq_ray* rays, uint32_t n, uint32_t flags,
                  uint32_t cull_mask, rq_hit* hits, rq_stream stream);
int rq_tlas_destroy(rq_tlas* tlas);

/* Launch shapes of a batch's two kernels.  Results do not depend on them. */
typedef struct rq_batch_tuning {
    uint32_t build_threads;       /* threads per build block: 256, 512 or 1024 */
    uint32_t build_blocks;        /* persistent build blocks (clamped to max_build_blocks) */
    uint32_t trace_threads;       /* threads per traversal block: 64, 128 or 256 */
    uint32_t trace_chunk;         /* ray ids a warp takes per refill: 32 or 64 */
    uint32_t trace_reg_cap;       /* registers per thread the launch bounds allow: 0 (none), 64, 72
                                     (threads 64 or 128 only) or 80 */
    uint32_t trace_blocks_per_sm; /* 0: as many as fit */
    uint32_t stack_entries;       /* stack entries per lane; 0 or anything below
                                     3 * (depth + 2) + 1 means that bound */
    uint32_t max_build_blocks;    /* read only: build scratch slices the batch holds */
    float build_ms;               /* rq_batch_autotune: measured time of this shape */
    float trace_ms;
    uint32_t trace_refill_min;    /* idle lanes of a traversal warp get new rays once at least this
                                     many of 32 are idle (or all are): 1..32; 0 means 1 */
    uint32_t build_cluster;       /* build blocks per thread-block cluster: 0 or 1 (none), 2 or 4;
                                     a cluster builds one large mesh with all its blocks */
    uint32_t cluster_min_tris;    /* meshes of at least this many triangles are built by a whole
                                     cluster (build_cluster > 1), the others by single blocks */
} rq_batch_tuning;

int rq_batch_tuning_get(const rq_batch* batch, rq_batch_tuning* out);
/* Validates the shape (RQ_ERR_INVALID_ARG for one that has no kernel). */
int rq_batch_tuning_set(rq_batch* batch, const rq_batch_tuning* t);
/* Autotuner: builds the batch and traces the given rays once per candidate
 * shape — every build block size with 1..occupancy blocks per SM, clusters
 * of 2 and 4 blocks of 512 and 1,024 threads for the meshes of at least
 * 8,192 or 32,768 triangles, every
 * traversal block size x refill chunk x register cap, then refill thresholds
 * for the fastest traversal shape — timing each with CUDA events (median of
 * `reps`), and keeps the fastest build and traversal shape.
 * The stack depth is the smallest safe one for the batch's deepest tree.
 * Writes up to `cap` measured candidates to `trials` (build_ms set for build
 * shapes, trace_ms for traversal shapes) and their number to *count.
 * Synchronous; overwrites the batch and `hits`. */
int rq_batch_autotune(rq_ctx* ctx, rq_batch* batch, const float* positions, uint32_t stride_bytes,
                      const uint32_t* indices, const rq_ray* rays, const uint32_t* ray_mesh,
                      const uint32_t* ray_flags, uint32_t n, rq_hit* hits, uint32_t reps, rq_batch_tuning* trials,
                      uint32_t cap, uint32_t* count, rq_stream stream);

/* ------------------------------------------------------------------ */
/* Frames: rays generated inside the traversal kernels                 */
/* ------------------------------------------------------------------ */

/* Pinhole camera of benchmarks/exp1_visbuf/shaders/visbuf_raycast.comp:15-51:
 * pixel (x, y) looks through NDC ((x+jx)/W*2-1, (y+jy)/H*2-1, 1) mapped to
 * the world by inv_view_proj (column-major, GLSL convention) and divided by
 * w; the ray leaves cam_pos toward that point.  jx = jy = 0.5 without
 * jitter; with jitter they are per-pixel U(0,1) draws from `seed`. */
typedef struct rq_camera {
    float inv_view_proj[16];
    float cam_pos[3];
    uint32_t width;
    uint32_t height;
    uint32_t jitter;
    uint32_t seed;
    float tmin; /* 0.01 in visbuf_raycast.comp:295 */
    float tmax; /* 10000 in visbuf_raycast.comp:297 */
    uint32_t flags; /* RQ_TRI_* */
} rq_camera;

/* One G-buffer pixel (32 B): hit position, visibility value (primitive
 * id + 1, 0 for a miss, as visbuf_raycast.comp:304-310 writes it), unit face
 * normal turned toward the camera (rq_ao.comp:67-68), hit distance. */
typedef struct rq_gbuffer_px {
    float pos[3];
    uint32_t vis;
    float nrm[3];
    float t;
} rq_gbuffer_px;

typedef struct rq_light {
    float pos[3];
    float radius;
} rq_light;

#define RQ_MAX_LIGHTS 32

/* Shadow and ambient-occlusion parameters.  Per pixel with a hit, light k
 * casts an any-hit shadow ray when dist in [0.001, radius] and N.L > 0, from
 * P + shadow_bias*N with [shadow_tmin, dist - shadow_bias]
 * (shaders/tiled_lighting_ra.comp:118-148); ao_spp cosine-weighted any-hit
 * rays from P + ao_bias*N with [ao_tmin, ao_tmax], seeded y*W + x + 5544
 * (shaders/rq_ao.comp:18-94). */
typedef struct rq_shade_params {
    uint32_t width;
    uint32_t height;
    uint32_t num_lights; /* <= RQ_MAX_LIGHTS */
    uint32_t ao_spp;     /* 0: no AO rays (ao gets 1.0) */
    float ao_tmax;       /* maxAoDistance */
    float ao_tmin;       /* 0.01 */
    float ao_bias;       /* 0.03 */
    float shadow_tmin;   /* 0.01 */
    float shadow_bias;   /* 0.04 */
    uint32_t flags;      /* RQ_TRI_* */
    rq_light lights[RQ_MAX_LIGHTS];
} rq_shade_params;

/* Camera from eye / target / up (right-handed look-at), vertical field of
 * view in degrees and image size: fills inv_view_proj (Vulkan clip space,
 * y flipped as the reference's projection) and cam_pos; jitter off, tmin
 * 0.01, tmax 10000, watertight triangles.  Host only. */
int rq_camera_look_at(const float eye[3], const float target[3], const float up[3], float fovy_deg,
                      uint32_t width, uint32_t height, rq_camera* out);

/* Primary closest-hit rays for every pixel into `gbuf` (width*height
 * entries, device).  The visibility-buffer pass of visbuf_raycast.comp and
 * the G-buffer the lighting passes read.  `cam` is a host pointer. */
int rq_render_gbuffer(rq_ctx* ctx, const rq_bvh* bvh, const rq_camera* cam, rq_gbuffer_px* gbuf, rq_stream stream);

/* params->flags bit: also count node and triangle tests into counters[1..2] */
#define RQ_SHADE_COUNT_TESTS 16u

/* Shadow and AO rays for every G-buffer pixel, generated and traced in one
 * kernel.  light_mask[p] bit k = light k cast a shadow ray that reached it;
 * ao[p] = unoccluded fraction (1.0 for empty pixels).  `counters` (device,
 * may be NULL) accumulates [0] rays cast and, with RQ_SHADE_COUNT_TESTS,
 * [1] box tests (4 per node visited) and [2] triangle tests.  `params` is a
 * host pointer; the other buffers are device pointers. */
int rq_render_shadow_ao(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_shade_params* params,
                        uint32_t* light_mask, float* ao, unsigned long long* counters, rq_stream stream);

/* Reflection rays of shaders/tiled_lighting_ra.comp:91-113: per G-buffer
 * pixel with a hit, R = reflect(normalize(P - cam_pos), N) (GLSL reflect,
 * I - 2 dot(N, I) N, not renormalised) from P + bias*N over [tmin, tmax],
 * closest hit with gl_RayFlagsOpaqueEXT semantics. */
typedef struct rq_reflect_params {
    uint32_t width;
    uint32_t height;
    float cam_pos[3];
    float tmin;     /* 0.02 */
    float tmax;     /* 100 */
    float bias;     /* 0.04 */
    uint32_t flags; /* RQ_TRI_* */
} rq_reflect_params;

/* Closest-hit reflection ray of every G-buffer pixel into hits[p] (rq_hit:
 * hit, t, instance id 0, original primitive id; t = -1 and ids 0xFFFFFFFF
 * for a miss and for pixels that saw no geometry, whose reflection the
 * shader skips).  The lighting pass reads only hit / miss (:111-113); the
 * full record is kept for callers that shade the reflected surface.
 * `params` is a host pointer; gbuf and hits are device pointers. */
int rq_render_reflect(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_reflect_params* params,
                      rq_hit* hits, rq_stream stream);

/* Ambient occlusion from a depth buffer, as shaders/rq_ao.comp:47-97 computes
 * it: per pixel (x, y), uv = ((x, y) + 0.5) / (W, H); depth >= 1 gives
 * AO = 1; otherwise the world position is inv_view_proj * (uv*2-1, depth, 1)
 * divided by w, and the normal is the normalised cross product of the right
 * and upper neighbours' reconstructed positions minus it (uv + one texel,
 * depth read at the neighbouring pixel, clamped to the image edge as a
 * clamp-to-edge sampler at texel centres reads it), turned toward cam_pos.
 * max(1, spp) cosine-hemisphere any-hit rays (seed y*W + x + 5544) leave
 * P + bias*N over [tmin, max_distance]; AO = the unoccluded fraction. */
typedef struct rq_ao_depth_params {
    float inv_view_proj[16]; /* column-major, Vulkan [0,1] depth */
    float cam_pos[3];
    uint32_t width;
    uint32_t height;
    uint32_t spp;        /* samplesPerPixel */
    float max_distance;  /* maxAoDistance */
    float tmin;          /* 0.01 */
    float bias;          /* 0.03 */
    uint32_t flags;      /* RQ_TRI_* */
} rq_ao_depth_params;

/* rq_ao.comp's AO pass over a width x height depth buffer (device, e.g. the
 * output of rq_gbuffer_depth) into ao (device, width*height floats).
 * `counters` (device, may be NULL) accumulates [0] rays cast.  `params` is a
 * host pointer.  At most 32 samples per pixel. */
int rq_render_ao_depth(rq_ctx* ctx, const rq_bvh* bvh, const float* depth, const rq_ao_depth_params* params, float* ao,
                       unsigned long long* counters, rq_stream stream);

/* Depth z/w of every G-buffer position under the view-projection `view_proj`
 * (column-major, Vulkan [0,1] depth; 1.0 for pixels that saw no geometry),
 * the depth the AO blur compares.  Device pointers, npix pixels. */
int rq_gbuffer_depth(rq_ctx* ctx, const rq_gbuffer_px* gbuf, uint32_t npix, const float view_proj[16], float* depth,
                     rq_stream stream);
/* One pass of the depth-aware separable AO blur of shaders/bilateral_blur.comp:
 * a 9-tap Gaussian along (dir_x, dir_y) = (1, 0) or (0, 1), taps whose depth
 * differs from the centre's by depth_threshold or more dropped, pixels at
 * depth >= 1 passed through; taps clamped to the image edge.  w x h floats,
 * device pointers, out must not alias in.  Run twice (horizontal, vertical)
 * for the full blur. */
int rq_blur_ao(rq_ctx* ctx, const float* ao_in, const float* depth, float* ao_out, uint32_t width, uint32_t height,
               int dir_x, int dir_y, float depth_threshold, rq_stream stream);

/* ------------------------------------------------------------------ */
/* RADV image (fast_bvh_builder.comp)                                  */
/* ------------------------------------------------------------------ */

/* compute_tree_layout (include/radv_bvh.hpp:193-215).  Host only. */
int rq_radv_layout_get(uint32_t num_triangles, rq_radv_layout* out);
/* Bytes of the image: 192 + 128*boxes + 64*triangles. */
uint64_t rq_radv_size(uint32_t num_triangles);

/* Write the RADV image of shaders/fast_bvh_builder.comp:91-257 for any
 * triangle count: 64-B triangle nodes in input order, Box32 leaves over 4
 * consecutive triangles, bottom-up Box32 levels, the 136-B header and the
 * two pre-root dwords.  `tri9`: 9 floats per triangle (device).  Byte-identical
 * to the shader's output wherever the shader is defined (N <= 4096).
 * RQ_ERR_SIZE if as_bytes < rq_radv_size(num_triangles). */
int rq_build_radv(rq_ctx* ctx, const float* tri9, uint32_t num_triangles, void* as_image,
                  uint64_t as_bytes, rq_stream stream);

/* Refit an image built by rq_build_radv (or a refit) after the vertices moved,
 * with the triangle count unchanged — the driver's refit of the same
 * acceleration structure (common/vk_bvh.cpp:558-611).  The fast builder's
 * topology depends only on the triangle count (four consecutive triangles
 * per leaf box, four consecutive children per parent), so the refit keeps
 * it and rewrites the triangle nodes, every box and the header's total box:
 * the bytes equal rq_build_radv's on the new vertices.  The image's header
 * must describe num_triangles; if not, the image is rebuilt all the same and
 * the next rq_ctx_check reports RQ_ERR_STATE. */
int rq_refit_radv(rq_ctx* ctx, const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                  rq_stream stream);

/* Allocation-free variant of rq_build_radv, with no counterpart in the
 * reference.  For callers that own all of their device memory and cannot let
 * a library call cudaMalloc/cudaFree (which synchronise the device and can
 * fail under a fixed budget): it takes no context, allocates nothing, and
 * keeps its scratch in a static device array inside librq.so, so it accepts
 * at most RQ_RADV_NOALLOC_MAX_TRIANGLES triangles (RQ_ERR_UNSUPPORTED
 * beyond).  Runs on the current device.  Every call looks up the array's
 * device address there (cudaGetSymbolAddress, which allocates nothing); the
 * first call on a device, and the first after a device reset, also loads the
 * library's device code, so make that first call before any stream capture.
 * All calls share the one array: calls that overlap on the GPU race, so
 * order them on one stream.  tri9 must be 4-byte and as_image 16-byte
 * aligned (RQ_ERR_INVALID_ARG).  Output bytes equal rq_build_radv's. */
#define RQ_RADV_NOALLOC_MAX_TRIANGLES (1u << 24)
int rq_build_radv_noalloc(const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                          rq_stream stream);

/* Text description of a RADV image in host memory: the header, the root node's
 * children and, if child 0 is a triangle, that node — the text of the
 * reference's decoder dump_bvh_structure (include/radv_bvh.hpp:311-390).
 * Writes at most `capacity` bytes (NUL-terminated) and the full length to
 * *length; text may be NULL with capacity 0 to ask for the length.
 * RQ_ERR_SIZE when the text was cut. */
int rq_radv_describe(const void* host_image, uint64_t bytes, char* text, uint64_t capacity, uint64_t* length);

/* Device-side decode of a whole RADV image (every Box32 node, every child
 * reference, every triangle node) with its invariants counted: child ids
 * that leave their region, child boxes that differ from the child's own
 * bounds, nodes or triangle ids referenced other than exactly once.  Reads
 * are range-checked, so a damaged image is reported, not dereferenced.
 * Synchronous. */
typedef struct rq_radv_check {
    uint32_t header_ok;            /* header offsets and counts fit the image */
    uint32_t reserved;
    uint64_t box_nodes;            /* from the header */
    uint64_t triangle_nodes;
    uint64_t box_children;         /* valid Box32 child references found */
    uint64_t triangle_children;    /* valid triangle child references found */
    uint64_t bad_offsets;          /* child ids outside their region or stride, or of another type */
    uint64_t bad_boxes;            /* child boxes unequal to the child's bounds */
    uint64_t box_refs_wrong;       /* box nodes referenced other than once (the root: never) */
    uint64_t triangle_refs_wrong;  /* triangle nodes referenced other than once */
    uint64_t ids_wrong;            /* triangle ids 0..N-1 not present exactly once */
} rq_radv_check;
int rq_radv_validate(rq_ctx* ctx, const void* as_image, uint64_t as_bytes, rq_radv_check* out, rq_stream stream);

/* Trace rays through a RADV image (the rayQueryEXT role of
 * shaders/verify_rayquery.comp:41-59): primitive IDs are the nodes'
 * triangle_id; `bary` as in rq_trace. */
int rq_trace_radv(rq_ctx* ctx, const void* as_image, uint64_t as_bytes, const rq_ray* rays,
                  uint32_t n, uint32_t flags, rq_hit* hits, float* bary, rq_stream stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* RQ_H */
