// capi.cpp — the C ABI of include/rq.h: argument checks, context and handle
// lifetime, scratch management, and the calls into the kernel launchers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "rq_internal.h"

int rq_collapse_blocks(int device, int num_sms);
int rq_launch_analyze4(rq_ctx* ctx, rq_bvh* bvh, cudaStream_t st);
int rq_launch_analyze2(rq_ctx* ctx, rq_bvh* bvh, cudaStream_t st);

namespace {

inline cudaStream_t S(rq_stream s) { return static_cast<cudaStream_t>(s); }

int sync_counts(rq_bvh* b) {
    if (!b->ctx) return RQ_ERR_STATE;
    cudaError_t e = cudaStreamSynchronize(b->last_stream);
    if (e == cudaSuccess) e = cudaMemcpy(b->h_counts, b->d_counts, sizeof(b->h_counts), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return rq_cuda_status(b->ctx, e, "reading BVH counts");
    b->counts_valid = true;
    return RQ_OK;
}

void free_arrays(rq_bvh* b) {
    if (b->mem) cudaFree(b->mem);
    b->mem = nullptr;
    b->mem_bytes = 0;
    b->nodes2 = nullptr;
    b->tris = nullptr;
    b->perm = nullptr;
    b->skeys = nullptr;
    b->nodes4 = nullptr;
    b->map4 = nullptr;
    b->d_counts = nullptr;
    b->capacity = 0;
}

}  // namespace

// Bytes of the one allocation behind a handle: capacity N triangles,
// node2_cap binary nodes, node4_cap 4-wide nodes.
size_t rq_bvh_alloc_bytes(uint32_t n, uint32_t node2_cap, uint32_t node4_cap) {
    Carve c{0, 0};
    c.take<rq_bvh2_node>(node2_cap);
    c.take<rq_triangle>(n);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n);
    c.take<rq_bvh4_node>(node4_cap);
    c.take<int32_t>(4ull * node4_cap);
    c.take<uint32_t>(4);
    return c.off + 256;
}

namespace {

// One allocation carved into the layouts.
int alloc_arrays(rq_ctx* ctx, rq_bvh* b, uint32_t n, uint32_t node2_cap, uint32_t node4_cap) {
    size_t bytes = rq_bvh_alloc_bytes(n, node2_cap, node4_cap);
    void* mem = nullptr;
    cudaError_t e = cudaMalloc(&mem, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return rq_set_error(ctx, RQ_ERR_OOM, "BVH allocation of " + std::to_string(bytes) + " bytes failed");
    }
    Carve d{reinterpret_cast<uintptr_t>(mem), 0};
    b->nodes2 = d.take<rq_bvh2_node>(node2_cap);
    b->tris = d.take<rq_triangle>(n);
    b->perm = d.take<uint32_t>(n);
    b->skeys = d.take<uint32_t>(n);
    b->nodes4 = d.take<rq_bvh4_node>(node4_cap);
    b->map4 = d.take<int32_t>(4ull * node4_cap);
    b->d_counts = d.take<uint32_t>(4);
    b->mem = mem;
    b->mem_bytes = bytes;
    b->capacity = n;
    b->cap_nodes2 = node2_cap;
    b->cap_nodes4 = node4_cap;
    cudaMemset(b->d_counts, 0, 4 * sizeof(uint32_t));
    return RQ_OK;
}

const char* kStatusText[] = {"ok",
                             "invalid argument",
                             "buffer too small",
                             "CUDA error",
                             "out of device memory",
                             "bounded device wait timed out",
                             "unsupported input",
                             "memory budget exceeded",
                             "no sm_100 device",
                             "handle not built",
                             "request cancelled"};

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace

// ---------------------------------------------------------------- internals

int rq_set_error(rq_ctx* ctx, int status, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    return status;
}

int rq_cuda_status(rq_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaSuccess) return RQ_OK;
    cudaGetLastError();
    int st = e == cudaErrorMemoryAllocation ? RQ_ERR_OOM : RQ_ERR_CUDA;
    return rq_set_error(ctx, st, std::string(what) + ": " + cudaGetErrorString(e));
}

int rq_ensure_scratch(rq_ctx* ctx, size_t bytes, cudaStream_t s) {
    if (ctx->scratch_bytes >= bytes) return RQ_OK;
    // the old block may still be read by work queued on `s`
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "scratch resize sync");
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    size_t want = std::max(bytes + bytes / 4, size_t(1) << 20);
    e = cudaMalloc(&ctx->scratch, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->scratch = nullptr;
        return rq_set_error(ctx, RQ_ERR_OOM, "scratch allocation of " + std::to_string(want) + " bytes failed");
    }
    ctx->scratch_bytes = want;
    return RQ_OK;
}

// ---------------------------------------------------------------- context

extern "C" {

int rq_ctx_create(int device, rq_ctx** out) {
    if (!out) return RQ_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return RQ_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return RQ_ERR_NO_DEVICE;
    rq_ctx* ctx = new (std::nothrow) rq_ctx();
    if (!ctx) return RQ_ERR_OOM;
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    cudaSetDevice(device);
    if (cudaMalloc(&ctx->d_err, 256) != cudaSuccess || cudaMallocHost(&ctx->h_err, 256) != cudaSuccess ||
        cudaMalloc(&ctx->d_ctr, 256) != cudaSuccess) {
        cudaGetLastError();
        rq_ctx_destroy(ctx);
        return RQ_ERR_OOM;
    }
    cudaMemset(ctx->d_err, 0, 256);
    ctx->collapse_blocks = rq_collapse_blocks(device, ctx->num_sms);
    *out = ctx;
    return RQ_OK;
}

int rq_ctx_destroy(rq_ctx* ctx) {
    if (!ctx) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->d_err) cudaFree(ctx->d_err);
    if (ctx->d_ctr) cudaFree(ctx->d_ctr);
    if (ctx->h_err) cudaFreeHost(ctx->h_err);
    delete ctx;
    return RQ_OK;
}

const char* rq_status_string(int status) {
    if (status < 0 || status > RQ_ERR_CANCELLED) return "unknown status";
    return kStatusText[status];
}

const char* rq_ctx_last_error(const rq_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int rq_ctx_check(rq_ctx* ctx, rq_stream stream) {
    if (!ctx) return RQ_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(S(stream));
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "stream synchronize");
    e = cudaMemcpy(ctx->h_err, ctx->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "reading device error word");
    uint32_t w = ctx->h_err[0];
    if (!w) return RQ_OK;
    cudaMemset(ctx->d_err, 0, sizeof(uint32_t));
    if (w == RQ_DERR_STACK)
        return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "traversal stack too small for the tree's live depth");
    if (w == RQ_DERR_RADV_IMAGE)
        return rq_set_error(ctx, RQ_ERR_STATE, "rq_refit_radv: the image was not built for this triangle count");
    return rq_set_error(ctx, RQ_ERR_DEVICE_TIMEOUT, "device error word 0x" + std::to_string(w));
}

uint64_t rq_ctx_scratch_bytes(const rq_ctx* ctx) { return ctx ? ctx->scratch_bytes : 0; }

int rq_debug_wait_timeout(rq_ctx* ctx, const uint32_t* flag, uint32_t limit, rq_stream stream) {
    if (!ctx || !flag || limit > (1u << 20)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad wait check");
    cudaSetDevice(ctx->device);
    return rq_launch_wait_check(ctx, flag, limit, S(stream));
}

int rq_ctx_trace_tuning_get(const rq_ctx* ctx, rq_trace_tuning* out) {
    if (!ctx || !out) return RQ_ERR_INVALID_ARG;
    *out = ctx->shade_shape;
    return RQ_OK;
}

int rq_ctx_trace_tuning_set(rq_ctx* ctx, const rq_trace_tuning* t) {
    if (!ctx || !t) return RQ_ERR_INVALID_ARG;
    if (!rq_shade_shape_ok(*t)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no traversal kernel for this shape");
    if (t->refill_min > 32) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "refill_min above 32");
    if (t->leaf_batch > 32) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "leaf_batch above 32");
    ctx->shade_shape = *t;
    if (ctx->shade_shape.refill_min == 0) ctx->shade_shape.refill_min = 1;
    return RQ_OK;
}

int rq_ctx_camera_tuning_get(const rq_ctx* ctx, rq_camera_tuning* out) {
    if (!ctx || !out) return RQ_ERR_INVALID_ARG;
    *out = ctx->camera;
    return RQ_OK;
}

int rq_ctx_camera_tuning_set(rq_ctx* ctx, const rq_camera_tuning* t) {
    if (!ctx || !t) return RQ_ERR_INVALID_ARG;
    if (t->engine > 1 || t->refill_min > 32 || t->leaf_batch > 32)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad camera schedule");
    ctx->camera = *t;
    if (ctx->camera.refill_min == 0) ctx->camera.refill_min = 1;
    if (ctx->camera.leaf_batch == 0) ctx->camera.leaf_batch = 32;
    return RQ_OK;
}

// ---------------------------------------------------------------- meshes

int rq_deform_wave(rq_ctx* ctx, const float* base, float* out, uint32_t num_vertices, float t, float amp,
                   float freq, rq_stream stream) {
    if (!ctx || !base || !out) return RQ_ERR_INVALID_ARG;
    return rq_launch_deform(ctx, base, out, num_vertices, t, amp, freq, S(stream));
}

int rq_deform_wave_step(rq_ctx* ctx, const float* base, float* out, uint32_t num_vertices, uint32_t* state, float dt,
                        float amp, float freq, rq_stream stream) {
    if (!ctx || !base || !out || !state) return RQ_ERR_INVALID_ARG;
    return rq_launch_deform_step(ctx, base, out, num_vertices, state, dt, amp, freq, S(stream));
}

// ---------------------------------------------------------------- build

int rq_build(rq_ctx* ctx, const float* positions, uint32_t stride_bytes, uint32_t num_vertices,
             const uint32_t* indices, uint32_t num_triangles, uint32_t max_leaf, uint32_t flags, rq_bvh** out,
             rq_stream stream) {
    if (!ctx || !positions || !out) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (num_triangles == 0) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no triangles");
    if (num_triangles >= RQ_MAX_TRIANGLES) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "more than 2^27 triangles");
    if (stride_bytes < 12 || stride_bytes % 4) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad vertex stride");
    if (max_leaf < 1 || max_leaf > 16) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "max_leaf must be 1..16");
    if (flags & ~(RQ_BUILD_BVH4 | RQ_BUILD_MEDIAN | RQ_BUILD_SAH))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "unknown build flags");
    if ((flags & RQ_BUILD_MEDIAN) && (flags & RQ_BUILD_SAH))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "RQ_BUILD_MEDIAN and RQ_BUILD_SAH exclude each other");
    if (!indices && uint64_t(num_vertices) < 3ull * num_triangles)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "non-indexed mesh needs 3 vertices per triangle");
    cudaSetDevice(ctx->device);
    rq_bvh* b = *out;
    bool fresh = false;
    if (b && (b->foreign || b->capacity < num_triangles || b->ctx != ctx)) {
        free_arrays(b);
        b->foreign = false;
        b->counts_valid = false;
    }
    if (!b) {
        b = new (std::nothrow) rq_bvh();
        if (!b) return RQ_ERR_OOM;
        fresh = true;
    }
    if (!b->mem) {
        b->ctx = ctx;
        b->device = ctx->device;
        int rc = alloc_arrays(ctx, b, num_triangles, 2 * num_triangles, std::max(1u, num_triangles));
        if (rc) {
            if (fresh) delete b;
            return rc;
        }
        b->counts_valid = false;
    }
    const bool want4 = (flags & RQ_BUILD_BVH4) != 0;
    int rc = (flags & RQ_BUILD_MEDIAN)
                 ? rq_launch_build_median(ctx, b, positions, stride_bytes, indices, num_triangles, max_leaf, want4,
                                          S(stream))
                 : rq_launch_build(ctx, b, positions, stride_bytes, indices, num_triangles, max_leaf, want4, S(stream),
                                   (flags & RQ_BUILD_SAH) ? RQ_SAH_SUBTREE_MAX : 0u);
    if (rc) {
        if (fresh) {
            free_arrays(b);
            delete b;
        }
        return rc;
    }
    b->num_tris = num_triangles;
    b->max_leaf = max_leaf;
    b->has4 = want4;
    b->built = true;
    b->last_stream = S(stream);
    *out = b;
    // a handle's first build reads the node counts back (one synchronisation);
    // in-place rebuilds stay asynchronous
    if (!b->counts_valid) return sync_counts(b);
    return RQ_OK;
}

int rq_collapse4(rq_ctx* ctx, rq_bvh* bvh, rq_stream stream) {
    if (!ctx || !bvh) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!bvh->built) return rq_set_error(ctx, RQ_ERR_STATE, "handle not built");
    cudaSetDevice(ctx->device);
    BuildScratch s;
    uint32_t n = std::max(bvh->capacity, bvh->cap_nodes2);
    size_t need = rq_build_scratch_carve(nullptr, n, s);
    int rc = rq_ensure_scratch(ctx, need, S(stream));
    if (rc) return rc;
    rq_build_scratch_carve(ctx->scratch, n, s);
    rc = rq_launch_collapse(ctx, bvh, s, S(stream));
    if (rc) return rc;
    bvh->has4 = true;
    bvh->last_stream = S(stream);
    if (bvh->foreign) {
        rc = rq_launch_analyze4(ctx, bvh, S(stream));
        if (rc) return rc;
    }
    return sync_counts(bvh);
}

int rq_refit(rq_ctx* ctx, rq_bvh* bvh, const float* positions, uint32_t stride_bytes, const uint32_t* indices,
             rq_stream stream) {
    if (!ctx || !bvh || !positions) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!bvh->built || bvh->foreign) return rq_set_error(ctx, RQ_ERR_STATE, "refit needs a handle built by rq_build");
    if (stride_bytes < 12 || stride_bytes % 4) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad vertex stride");
    cudaSetDevice(ctx->device);
    bvh->last_stream = S(stream);
    return rq_launch_refit(ctx, bvh, positions, stride_bytes, indices, S(stream));
}

static int import_common(rq_ctx* ctx, uint32_t num_nodes, const rq_triangle* tris, const uint32_t* perm,
                         uint32_t num_triangles, bool four, rq_bvh** out, rq_bvh** made) {
    if (!ctx || !out || !tris || num_nodes == 0 || num_triangles == 0)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad import arguments");
    if (num_triangles >= RQ_MAX_TRIANGLES) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "more than 2^27 triangles");
    cudaSetDevice(ctx->device);
    rq_bvh* b = new (std::nothrow) rq_bvh();
    if (!b) return RQ_ERR_OOM;
    b->ctx = ctx;
    b->device = ctx->device;
    b->foreign = true;
    uint32_t cap = std::max(num_triangles, num_nodes);
    int rc = alloc_arrays(ctx, b, cap, four ? 1u : num_nodes, four ? num_nodes : std::max(1u, num_nodes));
    if (rc) {
        delete b;
        return rc;
    }
    (void)perm;
    *made = b;
    return RQ_OK;
}

int rq_bvh_import2(rq_ctx* ctx, const rq_bvh2_node* nodes, uint32_t num_nodes, const rq_triangle* tris,
                   const uint32_t* perm, uint32_t num_triangles, rq_bvh** out, rq_stream stream) {
    if (!nodes) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null nodes");
    rq_bvh* b = nullptr;
    int rc = import_common(ctx, num_nodes, tris, perm, num_triangles, false, out, &b);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    cudaMemcpyAsync(b->nodes2, nodes, sizeof(rq_bvh2_node) * num_nodes, cudaMemcpyDefault, st);
    cudaMemcpyAsync(b->tris, tris, sizeof(rq_triangle) * num_triangles, cudaMemcpyDefault, st);
    if (perm) cudaMemcpyAsync(b->perm, perm, sizeof(uint32_t) * num_triangles, cudaMemcpyDefault, st);
    uint32_t h[4] = {num_nodes, 0, 0, 0};
    cudaMemcpyAsync(b->d_counts, h, sizeof(h), cudaMemcpyHostToDevice, st);
    if (!perm) b->perm = nullptr;
    b->num_tris = num_triangles;
    b->built = true;
    b->last_stream = st;
    rc = rq_launch_analyze2(ctx, b, st);
    if (rc == RQ_OK) rc = sync_counts(b);
    if (rc) {
        rq_bvh_destroy(b);
        return rc;
    }
    *out = b;
    return RQ_OK;
}

int rq_bvh_import4(rq_ctx* ctx, const rq_bvh4_node* nodes, uint32_t num_nodes, const rq_triangle* tris,
                   const uint32_t* perm, uint32_t num_triangles, rq_bvh** out, rq_stream stream) {
    if (!nodes) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null nodes");
    rq_bvh* b = nullptr;
    int rc = import_common(ctx, num_nodes, tris, perm, num_triangles, true, out, &b);
    if (rc) return rc;
    cudaStream_t st = S(stream);
    cudaMemcpyAsync(b->nodes4, nodes, sizeof(rq_bvh4_node) * num_nodes, cudaMemcpyDefault, st);
    cudaMemcpyAsync(b->tris, tris, sizeof(rq_triangle) * num_triangles, cudaMemcpyDefault, st);
    if (perm) cudaMemcpyAsync(b->perm, perm, sizeof(uint32_t) * num_triangles, cudaMemcpyDefault, st);
    uint32_t h[4] = {0, num_nodes, 0, 0};
    cudaMemcpyAsync(b->d_counts, h, sizeof(h), cudaMemcpyHostToDevice, st);
    if (!perm) b->perm = nullptr;
    b->num_tris = num_triangles;
    b->built = true;
    b->has4 = true;
    b->last_stream = st;
    rc = rq_launch_analyze4(ctx, b, st);
    if (rc == RQ_OK) rc = sync_counts(b);
    if (rc == RQ_OK && b->h_counts[3] > 16)
        rc = rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "leaf with more than 16 primitives");
    if (rc) {
        rq_bvh_destroy(b);
        return rc;
    }
    *out = b;
    return RQ_OK;
}

int rq_bvh_info_get(rq_bvh* bvh, rq_bvh_info* info) {
    if (!bvh || !info) return RQ_ERR_INVALID_ARG;
    if (!bvh->built) return RQ_ERR_STATE;
    cudaSetDevice(bvh->device);
    int rc = sync_counts(bvh);
    if (rc) return rc;
    info->num_triangles = bvh->num_tris;
    info->num_nodes2 = bvh->h_counts[0];
    info->num_nodes4 = bvh->has4 ? bvh->h_counts[1] : 0;
    info->depth4 = bvh->has4 ? bvh->h_counts[2] : 0;
    info->max_leaf = bvh->h_counts[3];
    info->stack_bound = bvh->has4 ? 3 * bvh->h_counts[2] + 1 : 0;
    info->device_bytes = bvh->mem_bytes;
    return RQ_OK;
}

int rq_bvh_download(rq_bvh* bvh, int host, rq_bvh2_node* nodes2, uint32_t cap_nodes2, rq_triangle* tris,
                    uint32_t cap_tris, rq_bvh4_node* nodes4, uint32_t cap_nodes4, uint32_t* perm, uint32_t cap_perm) {
    if (!bvh) return RQ_ERR_INVALID_ARG;
    if (!bvh->built) return RQ_ERR_STATE;
    cudaSetDevice(bvh->device);
    int rc = sync_counts(bvh);
    if (rc) return rc;
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    const uint32_t n2 = bvh->h_counts[0], n4 = bvh->has4 ? bvh->h_counts[1] : 0, nt = bvh->num_tris;
    if ((nodes2 && cap_nodes2 < n2) || (tris && cap_tris < nt) || (nodes4 && cap_nodes4 < n4) ||
        (perm && cap_perm < nt))
        return rq_set_error(bvh->ctx, RQ_ERR_SIZE, "download destination too small");
    cudaError_t e = cudaSuccess;
    if (nodes2 && n2 && e == cudaSuccess) e = cudaMemcpy(nodes2, bvh->nodes2, sizeof(rq_bvh2_node) * n2, k);
    if (tris && e == cudaSuccess) e = cudaMemcpy(tris, bvh->tris, sizeof(rq_triangle) * nt, k);
    if (nodes4 && n4 && e == cudaSuccess) e = cudaMemcpy(nodes4, bvh->nodes4, sizeof(rq_bvh4_node) * n4, k);
    if (perm && e == cudaSuccess) {
        if (bvh->perm) {
            e = cudaMemcpy(perm, bvh->perm, sizeof(uint32_t) * nt, k);
        } else if (host) {
            for (uint32_t i = 0; i < nt; ++i) perm[i] = i;
        } else {
            return rq_set_error(bvh->ctx, RQ_ERR_STATE, "imported handle has no permutation");
        }
    }
    return rq_cuda_status(bvh->ctx, e, "download");
}

int rq_bvh_download_sort(rq_bvh* bvh, int host, uint32_t* morton, uint32_t* sorted_ids, uint32_t cap) {
    if (!bvh) return RQ_ERR_INVALID_ARG;
    if (!bvh->built || bvh->foreign) return RQ_ERR_STATE;
    cudaSetDevice(bvh->device);
    int rc = sync_counts(bvh);
    if (rc) return rc;
    if (cap < bvh->num_tris) return rq_set_error(bvh->ctx, RQ_ERR_SIZE, "download destination too small");
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaSuccess;
    if (morton) e = cudaMemcpy(morton, bvh->skeys, sizeof(uint32_t) * bvh->num_tris, k);
    if (sorted_ids && e == cudaSuccess) e = cudaMemcpy(sorted_ids, bvh->perm, sizeof(uint32_t) * bvh->num_tris, k);
    return rq_cuda_status(bvh->ctx, e, "download sort");
}

int rq_bvh_destroy(rq_bvh* bvh) {
    if (!bvh) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(bvh->device);
    if (bvh->last_stream) cudaStreamSynchronize(bvh->last_stream);
    free_arrays(bvh);
    delete bvh;
    return RQ_OK;
}

// ---------------------------------------------------------------- trace

int rq_trace(rq_ctx* ctx, const rq_bvh* bvh, const rq_ray* rays, uint32_t n, uint32_t flags, rq_hit* hits,
             float* bary, rq_ray_stats* stats, rq_stream stream) {
    if (!ctx || !bvh || (n && (!rays || !hits))) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!bvh->built || !bvh->has4) return rq_set_error(ctx, RQ_ERR_STATE, "handle has no 4-wide BVH");
    if (flags & ~3u) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "unknown trace flags");
    if (!aligned(rays, 16) || !aligned(hits, 16) || (bary && !aligned(bary, 8)) || (stats && !aligned(stats, 16)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned ray/hit buffer");
    cudaSetDevice(ctx->device);
    if (!bvh->counts_valid) {
        int rc = sync_counts(const_cast<rq_bvh*>(bvh));
        if (rc) return rc;
    }
    if (bvh->h_counts[3] > 16) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "leaf with more than 16 primitives");
    return rq_launch_trace(ctx, bvh, rays, n, flags, hits, bary, stats, S(stream));
}

int rq_trace_ref_bvh4(rq_ctx* ctx, const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                      uint32_t n, rq_ray_stats* stats, rq_hit* hits, rq_stream stream) {
    if (!ctx || (n && (!nodes || !tris || !rays || (!stats && !hits))))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(ctx->device);
    return rq_launch_trace_ref4(ctx, nodes, tris, rays, n, stats, hits, S(stream));
}

int rq_trace_ref_bvh2(rq_ctx* ctx, const rq_bvh2_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                      uint32_t n, float t_eps, uint32_t* hit_flags, rq_stream stream) {
    if (!ctx || (n && (!nodes || !tris || !rays || !hit_flags)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(ctx->device);
    return rq_launch_trace_ref2(ctx, nodes, tris, rays, n, t_eps, hit_flags, S(stream));
}

int rq_gen_rays_procedural(rq_ctx* ctx, const float cam_pos[3], const float look_at[3], uint32_t count,
                           uint32_t coherent, rq_ray* rays, rq_stream stream) {
    if (!ctx || !cam_pos || !look_at || (count && !rays)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!aligned(rays, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned ray buffer");
    cudaSetDevice(ctx->device);
    return rq_launch_gen_procedural(ctx, cam_pos, look_at, count, coherent, rays, S(stream));
}

// ---------------------------------------------------------------- frames

static int frame_checks(rq_ctx* ctx, const rq_bvh* bvh) {
    if (!bvh->built || !bvh->has4) return rq_set_error(ctx, RQ_ERR_STATE, "handle has no 4-wide BVH");
    if (!bvh->counts_valid) {
        int rc = sync_counts(const_cast<rq_bvh*>(bvh));
        if (rc) return rc;
    }
    if (bvh->h_counts[3] > 16) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "leaf with more than 16 primitives");
    if (3u * bvh->h_counts[2] + 1u > 128u)
        return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "4-wide tree deeper than 42 levels");
    return RQ_OK;
}

int rq_render_gbuffer(rq_ctx* ctx, const rq_bvh* bvh, const rq_camera* cam, rq_gbuffer_px* gbuf, rq_stream stream) {
    if (!ctx || !bvh || !cam || !gbuf) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (cam->width == 0 || cam->height == 0 || (cam->flags & ~2u))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad camera");
    if (!aligned(gbuf, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned G-buffer");
    cudaSetDevice(ctx->device);
    int rc = frame_checks(ctx, bvh);
    if (rc) return rc;
    return rq_launch_gbuffer(ctx, bvh, *cam, gbuf, S(stream));
}

int rq_render_shadow_ao(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_shade_params* params,
                        uint32_t* light_mask, float* ao, unsigned long long* counters, rq_stream stream) {
    if (!ctx || !bvh || !gbuf || !params || !light_mask || !ao)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (params->num_lights > RQ_MAX_LIGHTS || params->ao_spp > 32 || params->width == 0 || params->height == 0 ||
        (params->flags & ~(RQ_TRI_MT | RQ_SHADE_COUNT_TESTS)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad shading parameters");
    if (!aligned(gbuf, 16) || (counters && !aligned(counters, 8)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned buffer");
    cudaSetDevice(ctx->device);
    int rc = frame_checks(ctx, bvh);
    if (rc) return rc;
    return rq_launch_shadow_ao(ctx, bvh, gbuf, *params, light_mask, ao, counters, S(stream));
}

int rq_render_reflect(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_reflect_params* params,
                      rq_hit* hits, rq_stream stream) {
    if (!ctx || !bvh || !gbuf || !params || !hits) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (params->width == 0 || params->height == 0 || (params->flags & ~RQ_TRI_MT))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad reflection parameters");
    if (!aligned(gbuf, 16) || !aligned(hits, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned buffer");
    cudaSetDevice(ctx->device);
    int rc = frame_checks(ctx, bvh);
    if (rc) return rc;
    return rq_launch_reflect(ctx, bvh, gbuf, *params, hits, S(stream));
}

int rq_render_ao_depth(rq_ctx* ctx, const rq_bvh* bvh, const float* depth, const rq_ao_depth_params* params, float* ao,
                       unsigned long long* counters, rq_stream stream) {
    if (!ctx || !bvh || !depth || !params || !ao) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (params->width == 0 || params->height == 0 || params->spp > 32 || (params->flags & ~RQ_TRI_MT))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad AO parameters");
    if (!aligned(depth, 4) || !aligned(ao, 4) || (counters && !aligned(counters, 8)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned buffer");
    cudaSetDevice(ctx->device);
    int rc = frame_checks(ctx, bvh);
    if (rc) return rc;
    return rq_launch_ao_depth(ctx, bvh, depth, *params, ao, counters, S(stream));
}

// ---------------------------------------------------------------- RADV

int rq_radv_layout_get(uint32_t n, rq_radv_layout* out) {
    if (!out) return RQ_ERR_INVALID_ARG;
    std::memset(out, 0, sizeof(*out));
    out->num_triangles = n;
    uint32_t counts[32];
    uint32_t lv = 0;
    counts[lv++] = (n + 3) / 4;
    while (counts[lv - 1] > 1) {
        if (lv >= 16) return RQ_ERR_UNSUPPORTED;
        counts[lv] = (counts[lv - 1] + 3) / 4;
        ++lv;
    }
    out->num_levels = lv;
    uint32_t off = 0;
    for (uint32_t i = 0; i < lv; ++i) {
        out->level_counts[i] = counts[lv - 1 - i];
        out->level_offsets[i] = off;
        off += out->level_counts[i];
    }
    out->total_boxes = off;
    out->total_as_size = 192ull + 128ull * off + 64ull * n;
    out->total_as_size_lo = uint32_t(out->total_as_size);
    return RQ_OK;
}

uint64_t rq_radv_size(uint32_t n) {
    rq_radv_layout l;
    if (rq_radv_layout_get(n, &l)) return 0;
    return l.total_as_size;
}

int rq_build_radv(rq_ctx* ctx, const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                  rq_stream stream) {
    if (!ctx || !tri9 || !as_image) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (num_triangles == 0) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no triangles");
    if (num_triangles > (1u << 25))
        return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "RADV node offsets are 32-bit: at most 2^25 triangles");
    if (!aligned(as_image, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "image must be 16-byte aligned");
    if (!aligned(tri9, 4)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "vertex buffer must be 4-byte aligned");
    rq_radv_layout L;
    if (rq_radv_layout_get(num_triangles, &L)) return RQ_ERR_UNSUPPORTED;
    if (as_bytes < L.total_as_size) return rq_set_error(ctx, RQ_ERR_SIZE, "image buffer smaller than rq_radv_size");
    cudaSetDevice(ctx->device);
    return rq_launch_radv(ctx, tri9, num_triangles, as_image, L, S(stream));
}

int rq_refit_radv(rq_ctx* ctx, const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                  rq_stream stream) {
    if (!ctx || !tri9 || !as_image) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (num_triangles == 0) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no triangles");
    if (num_triangles > (1u << 25))
        return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "RADV node offsets are 32-bit: at most 2^25 triangles");
    if (!aligned(as_image, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "image must be 16-byte aligned");
    if (!aligned(tri9, 4)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "vertex buffer must be 4-byte aligned");
    rq_radv_layout L;
    if (rq_radv_layout_get(num_triangles, &L)) return RQ_ERR_UNSUPPORTED;
    if (as_bytes < L.total_as_size) return rq_set_error(ctx, RQ_ERR_SIZE, "image buffer smaller than rq_radv_size");
    cudaSetDevice(ctx->device);
    return rq_launch_radv(ctx, tri9, num_triangles, as_image, L, S(stream), true);
}

int rq_trace_radv(rq_ctx* ctx, const void* as_image, uint64_t as_bytes, const rq_ray* rays, uint32_t n,
                  uint32_t flags, rq_hit* hits, float* bary, rq_stream stream) {
    if (!ctx || !as_image || (n && (!rays || !hits))) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (flags & ~3u) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "unknown trace flags");
    if (as_bytes < 192 + 128) return rq_set_error(ctx, RQ_ERR_SIZE, "image too small");
    if (!aligned(as_image, 16) || !aligned(rays, 16) || !aligned(hits, 16))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned buffer");
    cudaSetDevice(ctx->device);
    return rq_launch_trace_radv(ctx, as_image, as_bytes, rays, n, flags, hits, bary, S(stream));
}

int rq_gbuffer_depth(rq_ctx* ctx, const rq_gbuffer_px* gbuf, uint32_t npix, const float view_proj[16], float* depth,
                     rq_stream stream) {
    if (!ctx || (npix && (!gbuf || !depth)) || !view_proj) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!aligned(gbuf, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned G-buffer");
    cudaSetDevice(ctx->device);
    return rq_launch_gbuffer_depth(ctx, gbuf, npix, view_proj, depth, S(stream));
}

int rq_blur_ao(rq_ctx* ctx, const float* ao_in, const float* depth, float* ao_out, uint32_t width, uint32_t height,
               int dir_x, int dir_y, float depth_threshold, rq_stream stream) {
    if (!ctx || ((width && height) && (!ao_in || !depth || !ao_out)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!((dir_x == 1 && dir_y == 0) || (dir_x == 0 && dir_y == 1)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "blur direction must be (1,0) or (0,1)");
    if (ao_in == ao_out) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "blur output aliases its input");
    cudaSetDevice(ctx->device);
    return rq_launch_blur_ao(ctx, ao_in, depth, ao_out, width, height, dir_x, dir_y, depth_threshold, S(stream));
}

int rq_radv_validate(rq_ctx* ctx, const void* as_image, uint64_t as_bytes, rq_radv_check* out, rq_stream stream) {
    if (!ctx || !as_image || !out) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!aligned(as_image, 16)) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned image");
    cudaSetDevice(ctx->device);
    return rq_launch_radv_check(ctx, as_image, as_bytes, out, S(stream));
}

}  // extern "C"
