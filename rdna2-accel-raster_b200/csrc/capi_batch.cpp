// capi_batch.cpp — C ABI of batches (include/rq.h): many meshes in one
// allocation, built by one persistent launch and traced by one launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <string>
#include <vector>

#include "rq_batch.h"

namespace {

constexpr uint32_t kMaxBatchMeshTris = 1u << 20;
constexpr size_t kScratchBudget = size_t(4) << 30;  // per-block build scratch, all blocks

void free_batch(rq_batch* b) {
    if (b->mem) cudaFree(b->mem);
    if (b->scratch) cudaFree(b->scratch);
    b->mem = nullptr;
    b->scratch = nullptr;
}

int sync_batch_counts(rq_batch* b) {
    cudaError_t e = cudaStreamSynchronize(b->last_stream);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->h_counts.data(), b->d_counts, sizeof(uint32_t) * b->h_counts.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return rq_cuda_status(b->ctx, e, "reading batch counts");
    uint32_t md = 0;
    for (uint32_t m = 0; m < b->num_meshes; ++m) md = std::max(md, b->h_counts[4 * m + 2]);
    b->max_depth = md;
    b->counts_valid = true;
    return RQ_OK;
}

// Default shapes: 512-thread build blocks, as many as fit; 128-thread
// traversal blocks, 32-id refills, no register cap.
rq_batch_tuning default_tuning(rq_ctx* ctx, uint32_t slices) {
    rq_batch_tuning t{};
    t.build_threads = 512;
    t.build_blocks = std::min<uint32_t>(slices, uint32_t(ctx->num_sms) *
                                                    uint32_t(std::max(1, rq_batch_build_occupancy(512))));
    t.trace_threads = 128;
    t.trace_chunk = 32;
    t.trace_reg_cap = 0;
    t.trace_blocks_per_sm = 0;
    t.stack_entries = 0;
    t.max_build_blocks = slices;
    t.trace_refill_min = 1;
    t.build_cluster = 1;
    t.cluster_min_tris = 16384;
    return t;
}

// Median time of `reps` runs of f() on stream st (after one warm-up run).
template <class F>
int time_median(rq_ctx* ctx, cudaStream_t st, uint32_t reps, F&& f, float* ms) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess)
        return rq_cuda_status(ctx, cudaGetLastError(), "tuning events");
    std::vector<float> t;
    int rc = f();
    for (uint32_t r = 0; r < reps && rc == RQ_OK; ++r) {
        cudaEventRecord(a, st);
        rc = f();
        cudaEventRecord(b, st);
        if (rc == RQ_OK) {
            cudaError_t e = cudaEventSynchronize(b);
            float x = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&x, a, b);
            if (e != cudaSuccess) rc = rq_cuda_status(ctx, e, "tuning timing");
            t.push_back(x);
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (rc) return rc;
    std::sort(t.begin(), t.end());
    *ms = t.empty() ? 0.0f : t[t.size() / 2];
    return RQ_OK;
}

}  // namespace

extern "C" {

int rq_batch_tuning_get(const rq_batch* batch, rq_batch_tuning* out) {
    if (!batch || !out) return RQ_ERR_INVALID_ARG;
    *out = batch->tune;
    out->max_build_blocks = batch->build_slices;
    return RQ_OK;
}

int rq_batch_tuning_set(rq_batch* batch, const rq_batch_tuning* t) {
    if (!batch || !t) return RQ_ERR_INVALID_ARG;
    if ((t->build_threads != 256 && t->build_threads != 512 && t->build_threads != 1024) || t->build_blocks == 0 ||
        !rq_batch_trace_shape_ok(t->trace_threads, t->trace_chunk, t->trace_reg_cap) || t->stack_entries > 128 ||
        t->trace_refill_min > 32 || (t->build_cluster > 1 && t->build_cluster != 2 && t->build_cluster != 4))
        return rq_set_error(batch->ctx, RQ_ERR_INVALID_ARG, "no kernel for this batch shape");
    if (t->build_cluster > 1 && rq_batch_build_clusters(t->build_threads, t->build_cluster) < 1)
        return rq_set_error(batch->ctx, RQ_ERR_UNSUPPORTED, "no resident cluster of this build shape");
    const float bm = batch->tune.build_ms, tm = batch->tune.trace_ms;
    batch->tune = *t;
    batch->tune.build_ms = bm;
    batch->tune.trace_ms = tm;
    batch->tune.max_build_blocks = batch->build_slices;
    return RQ_OK;
}

int rq_batch_autotune(rq_ctx* ctx, rq_batch* batch, const float* positions, uint32_t stride_bytes,
                      const uint32_t* indices, const rq_ray* rays, const uint32_t* ray_mesh,
                      const uint32_t* ray_flags, uint32_t n, rq_hit* hits, uint32_t reps, rq_batch_tuning* trials,
                      uint32_t cap, uint32_t* count, rq_stream stream) {
    if (!ctx || !batch || !positions || !indices || (n && (!rays || !ray_mesh || !hits)) || (cap && !trials) ||
        !count)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    reps = std::max(1u, std::min(reps, 50u));
    *count = 0;
    int rc = rq_batch_build(ctx, batch, positions, stride_bytes, indices, stream);
    if (rc == RQ_OK && !batch->counts_valid) rc = sync_batch_counts(batch);
    if (rc) return rc;
    const rq_batch_tuning start = batch->tune;
    auto record = [&](const rq_batch_tuning& t) {
        if (*count < cap) trials[*count] = t;
        ++*count;
    };
    // build shapes
    rq_batch_tuning best_b = start;
    float best_bms = -1.0f;
    for (uint32_t bt : {256u, 512u, 1024u}) {
        const int occ = rq_batch_build_occupancy(bt);
        for (int k = 1; k <= occ; ++k) {
            rq_batch_tuning t = start;
            t.build_threads = bt;
            t.build_blocks = std::min<uint32_t>(batch->build_slices, uint32_t(ctx->num_sms) * uint32_t(k));
            t.build_cluster = 1;
            if (k > 1 && t.build_blocks == std::min<uint32_t>(batch->build_slices, uint32_t(ctx->num_sms) * (k - 1)))
                continue;  // clamped to the same grid as k - 1
            batch->tune = t;
            float ms = 0.0f;
            rc = time_median(ctx, st, reps,
                             [&] { return rq_launch_batch_build(ctx, batch, positions, stride_bytes, indices, st); },
                             &ms);
            if (rc) break;
            t.build_ms = ms;
            t.trace_ms = 0.0f;
            record(t);
            if (best_bms < 0.0f || ms < best_bms) {
                best_bms = ms;
                best_b = t;
            }
        }
        if (rc) break;
    }
    // clusters for the largest meshes, at full occupancy
    for (uint32_t bt : {512u, 1024u}) {
        if (rc) break;
        const int occ = rq_batch_build_occupancy(bt);
        for (uint32_t cl : {2u, 4u}) {
            if (rc || occ < 1 || rq_batch_build_clusters(bt, cl) < 1) continue;
            for (uint32_t min_tris : {8192u, 32768u}) {
                rq_batch_tuning t = start;
                t.build_threads = bt;
                t.build_blocks = std::min<uint32_t>(batch->build_slices, uint32_t(ctx->num_sms) * uint32_t(occ));
                t.build_cluster = cl;
                t.cluster_min_tris = min_tris;
                if (t.build_blocks < cl) continue;
                batch->tune = t;
                float ms = 0.0f;
                rc = time_median(ctx, st, reps,
                                 [&] { return rq_launch_batch_build(ctx, batch, positions, stride_bytes, indices, st); },
                                 &ms);
                if (rc) break;
                t.build_ms = ms;
                t.trace_ms = 0.0f;
                record(t);
                if (ms < best_bms) {
                    best_bms = ms;
                    best_b = t;
                }
            }
        }
    }
    // traversal shapes (on the batch as built)
    rq_batch_tuning best_t = start;
    float best_tms = -1.0f;
    if (rc == RQ_OK && n) {
        for (uint32_t tt : {64u, 128u, 256u})
            for (uint32_t chunk : {32u, 64u})
                for (uint32_t regs : {0u, 64u, 72u, 80u}) {
                    if (regs == 72u && tt == 256u) continue;  // same occupancy as 80 at 256 threads
                    rq_batch_tuning t = best_b;
                    t.trace_threads = tt;
                    t.trace_chunk = chunk;
                    t.trace_reg_cap = regs;
                    t.trace_blocks_per_sm = 0;
                    t.stack_entries = 0;
                    t.trace_refill_min = 1;
                    batch->tune = t;
                    float ms = 0.0f;
                    rc = time_median(ctx, st, reps,
                                     [&] {
                                         return rq_launch_batch_trace(ctx, batch, rays, ray_mesh, ray_flags, n, 0u,
                                                                      hits, nullptr, ctx->d_ctr, st);
                                     },
                                     &ms);
                    if (rc) break;
                    t.build_ms = 0.0f;
                    t.trace_ms = ms;
                    record(t);
                    if (best_tms < 0.0f || ms < best_tms) {
                        best_tms = ms;
                        best_t = t;
                    }
                }
        // refill thresholds for the fastest traversal shape
        const rq_batch_tuning shape = best_t;
        for (uint32_t refill : {8u, 12u, 16u, 20u}) {
            if (rc) break;
            rq_batch_tuning t = shape;
            t.trace_refill_min = refill;
            batch->tune = t;
            float ms = 0.0f;
            rc = time_median(ctx, st, reps,
                             [&] {
                                 return rq_launch_batch_trace(ctx, batch, rays, ray_mesh, ray_flags, n, 0u, hits,
                                                              nullptr, ctx->d_ctr, st);
                             },
                             &ms);
            if (rc) break;
            t.build_ms = 0.0f;
            t.trace_ms = ms;
            record(t);
            if (ms < best_tms) {
                best_tms = ms;
                best_t = t;
            }
        }
    }
    rq_batch_tuning fin = best_b;
    fin.trace_threads = best_t.trace_threads;
    fin.trace_chunk = best_t.trace_chunk;
    fin.trace_reg_cap = best_t.trace_reg_cap;
    fin.trace_blocks_per_sm = best_t.trace_blocks_per_sm;
    fin.trace_refill_min = best_t.trace_refill_min;
    fin.stack_entries = (3u * (batch->max_depth + 2u) + 1u + 3u) & ~3u;
    fin.build_ms = std::max(0.0f, best_bms);
    fin.trace_ms = std::max(0.0f, best_tms);
    fin.max_build_blocks = batch->build_slices;
    batch->tune = rc == RQ_OK ? fin : start;
    return rc;
}

int rq_batch_create(rq_ctx* ctx, const rq_mesh_desc* meshes, uint32_t num_meshes, uint32_t max_leaf,
                    rq_batch** out) {
    if (!ctx || !meshes || !out || num_meshes == 0) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad batch");
    if (max_leaf < 1 || max_leaf > 16) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "max_leaf must be 1..16");
    uint64_t end = 0;
    uint32_t maxt = 0;
    for (uint32_t m = 0; m < num_meshes; ++m) {
        const rq_mesh_desc& d = meshes[m];
        if (d.num_triangles == 0 || d.num_triangles > kMaxBatchMeshTris)
            return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "batch meshes need 1..2^20 triangles");
        end = std::max<uint64_t>(end, uint64_t(d.triangle_offset) + d.num_triangles);
        maxt = std::max(maxt, d.num_triangles);
    }
    if (end >= RQ_MAX_TRIANGLES) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "batch larger than 2^27 triangles");
    // triangle ranges must not overlap
    std::vector<uint32_t> ord(num_meshes);
    std::iota(ord.begin(), ord.end(), 0u);
    std::sort(ord.begin(), ord.end(),
              [&](uint32_t a, uint32_t b) { return meshes[a].triangle_offset < meshes[b].triangle_offset; });
    for (uint32_t i = 1; i < num_meshes; ++i) {
        const rq_mesh_desc& p = meshes[ord[i - 1]];
        if (uint64_t(p.triangle_offset) + p.num_triangles > meshes[ord[i]].triangle_offset)
            return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "overlapping triangle ranges");
    }
    cudaSetDevice(ctx->device);
    rq_batch* b = new (std::nothrow) rq_batch();
    if (!b) return RQ_ERR_OOM;
    b->ctx = ctx;
    b->device = ctx->device;
    b->num_meshes = num_meshes;
    b->total_tris = uint32_t(end);
    b->max_tris = maxt;
    b->max_leaf = max_leaf;
    b->meshes.assign(meshes, meshes + num_meshes);
    b->h_counts.assign(4ull * num_meshes, 0u);
    const size_t T = end;
    Carve c{0, 0};
    c.take<rq_bvh2_node>(2 * T);
    c.take<rq_triangle>(T);
    c.take<uint32_t>(T);
    c.take<uint32_t>(T);
    c.take<rq_bvh4_node>(T);
    c.take<int32_t>(4 * T);
    c.take<uint32_t>(4ull * num_meshes);
    c.take<rq_mesh_desc>(num_meshes);
    c.take<uint32_t>(num_meshes);
    c.take<uint32_t>(64);
    b->mem_bytes = c.off + 256;
    b->scratch_stride = rq_batch_block_scratch(maxt);
    // scratch slices: enough for the most resident build blocks of any
    // block size, within the scratch budget and the mesh count
    int occ = 0;
    for (uint32_t t : {256u, 512u, 1024u}) occ = std::max(occ, rq_batch_build_occupancy(t));
    uint32_t blocks = uint32_t(ctx->num_sms) * uint32_t(std::max(1, occ));
    blocks = std::min<uint32_t>(blocks, uint32_t(std::max<size_t>(1, kScratchBudget / b->scratch_stride)));
    blocks = std::max(1u, std::min(blocks, num_meshes));
    b->build_slices = blocks;
    b->tune = default_tuning(ctx, blocks);
    if (cudaMalloc(&b->mem, b->mem_bytes) != cudaSuccess ||
        cudaMalloc(&b->scratch, b->scratch_stride * b->build_slices) != cudaSuccess) {
        cudaGetLastError();
        free_batch(b);
        delete b;
        return rq_set_error(ctx, RQ_ERR_OOM, "batch allocation failed");
    }
    Carve d{reinterpret_cast<uintptr_t>(b->mem), 0};
    b->nodes2 = d.take<rq_bvh2_node>(2 * T);
    b->tris = d.take<rq_triangle>(T);
    b->perm = d.take<uint32_t>(T);
    b->skeys = d.take<uint32_t>(T);
    b->nodes4 = d.take<rq_bvh4_node>(T);
    b->map4 = d.take<int32_t>(4 * T);
    b->d_counts = d.take<uint32_t>(4ull * num_meshes);
    b->d_meshes = d.take<rq_mesh_desc>(num_meshes);
    b->d_order = d.take<uint32_t>(num_meshes);
    b->d_ctr = d.take<uint32_t>(64);
    // build order: largest first, so the long builds start early
    std::vector<uint32_t> order(num_meshes);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t c2) {
        return meshes[a].num_triangles > meshes[c2].num_triangles;
    });
    cudaError_t e = cudaMemcpy(b->d_meshes, meshes, sizeof(rq_mesh_desc) * num_meshes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(b->d_order, order.data(), sizeof(uint32_t) * num_meshes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->d_counts, 0, sizeof(uint32_t) * 4 * num_meshes);
    if (e != cudaSuccess) {
        free_batch(b);
        delete b;
        return rq_cuda_status(ctx, e, "batch setup");
    }
    *out = b;
    return RQ_OK;
}

int rq_batch_build(rq_ctx* ctx, rq_batch* batch, const float* positions, uint32_t stride_bytes,
                   const uint32_t* indices, rq_stream stream) {
    if (!ctx || !batch || !positions || !indices) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (stride_bytes < 12 || stride_bytes % 4) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad vertex stride");
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = rq_launch_batch_build(ctx, batch, positions, stride_bytes, indices, st);
    if (rc) return rc;
    batch->built = true;
    batch->last_stream = st;
    if (!batch->counts_valid) return sync_batch_counts(batch);
    return RQ_OK;
}

int rq_batch_trace(rq_ctx* ctx, const rq_batch* batch, const rq_ray* rays, const uint32_t* ray_mesh,
                   const uint32_t* ray_flags, uint32_t n, uint32_t flags, rq_hit* hits, rq_ray_stats* stats,
                   rq_stream stream) {
    if (!ctx || !batch || (n && (!rays || !ray_mesh || !hits)))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (!batch->built) return rq_set_error(ctx, RQ_ERR_STATE, "batch not built");
    if (flags & ~3u) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "unknown trace flags");
    if (3u * batch->max_depth + 1u > 128u) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "4-wide tree too deep");
    if (n == 0) return RQ_OK;
    cudaSetDevice(ctx->device);
    return rq_launch_batch_trace(ctx, batch, rays, ray_mesh, ray_flags, n, flags, hits, stats, ctx->d_ctr,
                                 static_cast<cudaStream_t>(stream));
}

int rq_batch_info_get(rq_batch* batch, uint32_t mesh, rq_bvh_info* info) {
    if (!batch || !info || mesh >= batch->num_meshes) return RQ_ERR_INVALID_ARG;
    if (!batch->built) return RQ_ERR_STATE;
    cudaSetDevice(batch->device);
    int rc = sync_batch_counts(batch);
    if (rc) return rc;
    const uint32_t* c = &batch->h_counts[4ull * mesh];
    info->num_triangles = batch->meshes[mesh].num_triangles;
    info->num_nodes2 = c[0];
    info->num_nodes4 = c[1];
    info->depth4 = c[2];
    info->max_leaf = c[3];
    info->stack_bound = 3 * c[2] + 1;
    info->device_bytes = batch->mem_bytes;
    return RQ_OK;
}

int rq_batch_download(rq_batch* batch, uint32_t mesh, int host, rq_bvh2_node* nodes2, uint32_t cap_nodes2,
                      rq_triangle* tris, uint32_t cap_tris, rq_bvh4_node* nodes4, uint32_t cap_nodes4,
                      uint32_t* perm, uint32_t cap_perm) {
    rq_bvh_info inf;
    int rc = rq_batch_info_get(batch, mesh, &inf);
    if (rc) return rc;
    const size_t off = batch->meshes[mesh].triangle_offset;
    const uint32_t nt = inf.num_triangles;
    if ((nodes2 && cap_nodes2 < inf.num_nodes2) || (tris && cap_tris < nt) || (nodes4 && cap_nodes4 < inf.num_nodes4) ||
        (perm && cap_perm < nt))
        return rq_set_error(batch->ctx, RQ_ERR_SIZE, "download destination too small");
    const cudaMemcpyKind k = host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaSuccess;
    if (nodes2) e = cudaMemcpy(nodes2, batch->nodes2 + 2 * off, sizeof(rq_bvh2_node) * inf.num_nodes2, k);
    if (tris && e == cudaSuccess) e = cudaMemcpy(tris, batch->tris + off, sizeof(rq_triangle) * nt, k);
    if (nodes4 && e == cudaSuccess)
        e = cudaMemcpy(nodes4, batch->nodes4 + off, sizeof(rq_bvh4_node) * inf.num_nodes4, k);
    if (perm && e == cudaSuccess) e = cudaMemcpy(perm, batch->perm + off, sizeof(uint32_t) * nt, k);
    return rq_cuda_status(batch->ctx, e, "batch download");
}

int rq_batch_destroy(rq_batch* batch) {
    if (!batch) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(batch->device);
    if (batch->last_stream) cudaStreamSynchronize(batch->last_stream);
    free_batch(batch);
    delete batch;
    return RQ_OK;
}

}  // extern "C"
