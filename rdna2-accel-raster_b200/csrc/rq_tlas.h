// rq_tlas.h — host-side state of a two-level scene (rq_tlas) and the
// launchers of k_tlas.cu.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "rq_internal.h"

// Device record of one instance (80 B).
struct TlasInst {
    float inv[12];              // world -> object, row-major 3x4
    const rq_bvh4_node* nodes;  // the BLAS
    const rq_triangle* tris;
    const uint32_t* perm;
    uint32_t instance_id;
    uint32_t mask;
};
static_assert(sizeof(TlasInst) == 80, "TlasInst layout");

struct rq_tlas {
    rq_ctx* ctx = nullptr;
    int device = 0;
    uint32_t num_instances = 0;
    TlasInst* d_inst = nullptr;   // num_instances records
    float* d_fwd = nullptr;       // 12 floats per instance: object -> world
    float* d_tri9 = nullptr;      // the instances' world boxes as degenerate triangles
    rq_bvh* top = nullptr;        // BVH over the instance boxes, one instance per leaf
    uint32_t stack_bound = 0;     // entries per ray: top + marker + deepest BLAS
    cudaStream_t last_stream = nullptr;
};

int rq_launch_instance_boxes(rq_ctx* ctx, const TlasInst* inst, const float* fwd, uint32_t n, float* tri9,
                             cudaStream_t st);
int rq_launch_trace_tlas(rq_ctx* ctx, const rq_tlas* t, const rq_ray* rays, uint32_t n, uint32_t flags,
                         uint32_t cull_mask, rq_hit* hits, cudaStream_t st);
