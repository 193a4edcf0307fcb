// rq_batch.h — host-side state of a batch handle (many meshes, one
// allocation) and the launchers of k_batch.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "rq_internal.h"

struct rq_batch {
    rq_ctx* ctx = nullptr;
    int device = 0;
    uint32_t num_meshes = 0;
    uint32_t total_tris = 0;
    uint32_t max_tris = 0;
    uint32_t max_leaf = 4;
    std::vector<rq_mesh_desc> meshes;  // host copy
    // arrays of all meshes: mesh m's binary nodes start at 2*triangle_offset,
    // its triangles / permutation / keys / 4-wide nodes at triangle_offset
    void* mem = nullptr;
    size_t mem_bytes = 0;
    rq_bvh2_node* nodes2 = nullptr;
    rq_triangle* tris = nullptr;
    uint32_t* perm = nullptr;
    uint32_t* skeys = nullptr;
    rq_bvh4_node* nodes4 = nullptr;
    int32_t* map4 = nullptr;
    uint32_t* d_counts = nullptr;  // 4 per mesh: nodes2, nodes4, depth4, max leaf
    rq_mesh_desc* d_meshes = nullptr;
    uint32_t* d_order = nullptr;   // build order: largest mesh first
    uint32_t* d_ctr = nullptr;     // build queue counters: [0] clusters, [1] single blocks
    // per-block build scratch, sized for the largest mesh
    void* scratch = nullptr;
    size_t scratch_stride = 0;
    uint32_t build_slices = 0;     // scratch slices: the most build blocks a launch may use
    rq_batch_tuning tune{};        // launch shapes
    std::vector<uint32_t> h_counts;
    bool counts_valid = false;
    uint32_t max_depth = 0;
    bool built = false;
    cudaStream_t last_stream = nullptr;
};

size_t rq_batch_block_scratch(uint32_t max_tris);
// Resident build blocks per SM for a build block size (0 if none).
int rq_batch_build_occupancy(uint32_t threads);
// Resident clusters of `cluster` (2 or 4) build blocks of `threads` (0 if none).
int rq_batch_build_clusters(uint32_t threads, uint32_t cluster);
// Whether a traversal kernel exists for this shape.
bool rq_batch_trace_shape_ok(uint32_t threads, uint32_t chunk, uint32_t regs);
int rq_launch_batch_build(rq_ctx* ctx, rq_batch* b, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                          cudaStream_t st);
int rq_launch_batch_trace(rq_ctx* ctx, const rq_batch* b, const rq_ray* rays, const uint32_t* ray_mesh,
                          const uint32_t* ray_flags, uint32_t n, uint32_t flags, rq_hit* hits, rq_ray_stats* stats,
                          uint32_t* ctr, cudaStream_t st);
