// rq_internal.h — host-side internals of librq: context, BVH handle, scratch
// carving and the launchers each .cu file provides.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/rq.h"

// Device error word bits (rq_ctx::d_err), set by kernels whose bounded waits
// gave up; rq_ctx_check reports them as RQ_ERR_DEVICE_TIMEOUT.
#define RQ_DERR_SORT_LOOKBACK 1u
#define RQ_DERR_SCAN_LOOKBACK 2u
#define RQ_DERR_GRID_BARRIER 4u
#define RQ_DERR_REFIT 8u
#define RQ_DERR_STACK 16u
#define RQ_DERR_QUEUE 32u
#define RQ_DERR_WAIT_CHECK 64u
#define RQ_DERR_RADV_IMAGE 128u  // rq_refit_radv: the image's header is not for this triangle count

// Word of rq_ctx::d_err that holds the RADV build's finishing ticket: 0
// between launches, since the build's last block resets it.
#define RQ_CTX_RADV_TICKET 32

// Largest triangle count a leaf stack entry can address (27-bit first prim).
#define RQ_MAX_TRIANGLES (1u << 27)

struct rq_ctx {
    int device = 0;
    int num_sms = 0;
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    uint32_t* d_err = nullptr;      // device error word ([0]); 256 B, zeroed at creation
    uint32_t* h_err = nullptr;      // pinned mirror
    uint32_t* d_ctr = nullptr;      // work counters of persistent launches (zeroed per launch)
    std::string last_error;
    int collapse_blocks = 0;        // co-resident blocks of the collapse kernel
    rq_trace_tuning shade_shape{128, 32, 80, 0, 0, 1, 0};  // shadow/AO traversal launch shape
    rq_camera_tuning camera{0, 1, 32};                      // camera traversal schedule
};

struct rq_bvh {
    rq_ctx* ctx = nullptr;
    int device = 0;
    uint32_t capacity = 0;          // triangles the arrays can hold
    uint32_t num_tris = 0;
    uint32_t max_leaf = 4;
    bool has4 = false;
    bool built = false;
    bool foreign = false;           // imported arrays (no sort keys, no Karras data)
    rq_bvh2_node* nodes2 = nullptr; // capacity 2N
    rq_triangle* tris = nullptr;    // N
    uint32_t* perm = nullptr;       // N: leaf order -> original id
    uint32_t* skeys = nullptr;      // N: sorted Morton keys
    rq_bvh4_node* nodes4 = nullptr; // capacity max(1, N)
    int32_t* map4 = nullptr;        // 4 per 4-wide node: binary node of each slot (-1 empty)
    uint32_t cap_nodes2 = 0, cap_nodes4 = 0;
    uint32_t* d_counts = nullptr;   // [0] nodes2, [1] nodes4, [2] depth4, [3] max leaf count
    uint32_t h_counts[4] = {0, 0, 0, 0};
    bool counts_valid = false;
    cudaStream_t last_stream = nullptr;
    void* mem = nullptr;            // single allocation backing the arrays
    size_t mem_bytes = 0;
};

// Bump allocator over a scratch block (256-B aligned pieces).  With base 0
// it only measures.
struct Carve {
    uintptr_t base;
    size_t off = 0;
    template <class T>
    __host__ __device__ T* take(size_t n) {
        off = (off + 255) & ~size_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += n * sizeof(T);
        return p;
    }
};

int rq_set_error(rq_ctx* ctx, int status, const std::string& msg);
int rq_cuda_status(rq_ctx* ctx, cudaError_t e, const char* what);
// Make sure the context scratch holds at least `bytes`.
int rq_ensure_scratch(rq_ctx* ctx, size_t bytes, cudaStream_t s);

// ---------------------------------------------------------------- k_build
struct BuildScratch {
    float4* cent;          // N centroids (w unused)
    uint32_t* bounds;      // 6 ordered-uint: min xyz, max xyz
    uint32_t* keys[2];     // N each
    uint32_t* vals[2];     // N each
    uint32_t* hist;        // 4 x 256
    uint32_t* sort_status; // 4 passes x tiles x 256
    uint32_t* tile_ctr;    // 8 counters
    int32_t* kl;           // N-1 Karras left child (bit 31: leaf)
    int32_t* kr;           // N-1 right child
    uint32_t* klo;         // N-1 range start
    uint32_t* khi;         // N-1 range end (inclusive)
    uint32_t* par_in;      // N-1 parent of internal node: (parent << 1) | is_right
    uint32_t* par_lf;      // N   parent of leaf
    float4* box_in;        // 2(N-1): lo, hi
    float4* box_lf;        // 2N
    uint32_t* refit_flag;  // N-1
    uint32_t* c;           // N   emission counts
    uint32_t* a;           // N   exclusive scan of c
    uint32_t* scan_status; // tiles
    // collapse
    uint32_t* q;           // N queue of BVH2 node ids
    int32_t* cand;         // 4N candidates (BVH2 ids)
    int32_t* child_q;      // 4N queue index of inner children (-1 none)
    uint32_t* sz;          // N subtree sizes
    uint32_t* cpar;        // N parent link of each queue entry
    unsigned long long* cacc;  // N arrival counts and size sums
    uint32_t* coll_ctl;    // 256 words: [1] barrier count [2] barrier gen, [4..10] collapse control
    // LBVH with SAH-rebuilt subtrees (RQ_BUILD_SAH; null otherwise)
    uint32_t* sah_hi;      // N: at a subtree's first position, its last
    uint32_t* sah_L;       // N: at a subtree's first position, the left-child links above its root
    uint32_t* sah_node;    // N: at a subtree's first position, its root (bit 31: a Karras leaf)
    uint32_t* sah_list;    // N: first positions of the block subtrees (in the order they were found)
    uint32_t* sah_depth;   // N: at a block subtree's first position, its depth below its SAH root
    float4* sah_rec;       // 4N: two float4 per node record (box, first position, aux word)
    uint32_t* sah_rec_l;   // 2N: left-child links above the node, or kNoRecord for an unused slot
    float4* sah_plo;       // N: per sorted position, the triangle's box min and centroid x
    float4* sah_phi;       // N: box max and centroid y
    float* sah_pcz;        // N: centroid z
    uint32_t* sah_ord[2];  // N each: the order of the sorted positions at even / odd depths
    uint4* sah_mq;         // node queue of the nodes above a block's size: s, e, depth | L << 8, Karras node
    uint32_t* sah_mready;  // per queue entry: written
    float4* sah_mrec;      // two float4 per such node's record
    uint32_t* sah_mrec_l;  // left-child links above it
    uint32_t sah_mcap;     // capacity of the queue and of the records
    uint32_t* sah_ctl;     // 16 words: [0] queue head [1] queue tail [2] nodes done [3] records
};

// Carve the build scratch for n triangles out of `base`; returns its size
// (base may be null to measure).  sah: also the SAH-subtree arrays.
size_t rq_build_scratch_carve(void* base, uint32_t n, BuildScratch& s, bool sah = false);
// sah_max > 0: the LBVH above every node of at most sah_max triangles, each
// such subtree rebuilt by binned SAH (RQ_BUILD_SAH); 0: the plain LBVH.
int rq_launch_build(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                    uint32_t n, uint32_t max_leaf, bool collapse, cudaStream_t s, uint32_t sah_max = 0);
// The reference's median-split topology (k_median.cu); synchronises once per tree level.
int rq_launch_build_median(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                           uint32_t n, uint32_t max_leaf, bool collapse, cudaStream_t s);
int rq_launch_refit(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                    cudaStream_t s);

// ---------------------------------------------------------------- k_sort
uint32_t rq_sort_tiles(uint32_t n);
// Stable LSD radix sort of (keys, vals) on `bits` low key bits; result ends
// in buffer index returned (0 or 1).
int rq_launch_sort(rq_ctx* ctx, BuildScratch& s, uint32_t n, uint32_t bits, cudaStream_t st, int* result_buf);
uint32_t rq_scan_tiles(uint32_t n);
// Exclusive scan of in[0..n) (of in[order[i]] when order is given).
void rq_launch_scan(rq_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* status,
                    uint32_t* tile_ctr, cudaStream_t st, const uint32_t* order = nullptr);

// ---------------------------------------------------------------- k_collapse
int rq_launch_collapse(rq_ctx* ctx, rq_bvh* bvh, BuildScratch& s, cudaStream_t st);

// ---------------------------------------------------------------- k_trace
int rq_launch_trace(rq_ctx* ctx, const rq_bvh* bvh, const rq_ray* rays, uint32_t n, uint32_t flags, rq_hit* hits,
                    float* bary, rq_ray_stats* stats, cudaStream_t st);
int rq_launch_trace_ref4(rq_ctx* ctx, const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                         uint32_t n, rq_ray_stats* stats, rq_hit* hits, cudaStream_t st);
int rq_launch_trace_ref2(rq_ctx* ctx, const rq_bvh2_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                         uint32_t n, float t_eps, uint32_t* flags, cudaStream_t st);
int rq_launch_trace_radv(rq_ctx* ctx, const void* img, uint64_t bytes, const rq_ray* rays, uint32_t n,
                         uint32_t flags, rq_hit* hits, float* bary, cudaStream_t st);

// ---------------------------------------------------------------- k_frame
int rq_launch_gbuffer(rq_ctx* ctx, const rq_bvh* bvh, const rq_camera& cam, rq_gbuffer_px* gbuf, cudaStream_t st);
bool rq_shade_shape_ok(const rq_trace_tuning& t);
int rq_launch_shadow_ao(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_shade_params& p,
                        uint32_t* mask, float* ao, unsigned long long* counter, cudaStream_t st);
int rq_launch_reflect(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_reflect_params& p,
                      rq_hit* hits, cudaStream_t st);
int rq_launch_ao_depth(rq_ctx* ctx, const rq_bvh* bvh, const float* depth, const rq_ao_depth_params& p, float* ao,
                       unsigned long long* counters, cudaStream_t st);

// ---------------------------------------------------------------- k_radv
int rq_launch_radv(rq_ctx* ctx, const float* tri9, uint32_t n, void* img, const rq_radv_layout& L, cudaStream_t st,
                   bool refit = false);
int rq_launch_radv_check(rq_ctx* ctx, const void* img, uint64_t bytes, rq_radv_check* out, cudaStream_t st);

// ---------------------------------------------------------------- k_post
int rq_launch_gbuffer_depth(rq_ctx* ctx, const rq_gbuffer_px* gbuf, uint32_t npix, const float vp[16], float* depth,
                            cudaStream_t st);
int rq_launch_blur_ao(rq_ctx* ctx, const float* in, const float* depth, float* out, uint32_t w, uint32_t h, int dx,
                      int dy, float threshold, cudaStream_t st);

// ---------------------------------------------------------------- k_raygen
int rq_launch_gen_procedural(rq_ctx* ctx, const float cam[3], const float look[3], uint32_t count,
                             uint32_t coherent, rq_ray* rays, cudaStream_t st);
int rq_launch_deform(rq_ctx* ctx, const float* base, float* out, uint32_t nv, float t, float amp, float freq,
                     cudaStream_t st);
int rq_launch_wait_check(rq_ctx* ctx, const uint32_t* flag, uint32_t limit, cudaStream_t st);
int rq_launch_deform_step(rq_ctx* ctx, const float* base, float* out, uint32_t nv, uint32_t* state, float dt,
                          float amp, float freq, cudaStream_t st);
