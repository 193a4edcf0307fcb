// rq_serve_internal.h — the job table of a serving launch, shared by the
// host request loop (server.cpp) and the traversal kernel (k_serve.cu).
#pragma once

#include <cstdint>

#include "rq_internal.h"
#include "../../include/rq_serve.h"

// Most requests one launch carries (their id-space starts are staged in
// shared memory).
#define RQ_SERVE_MAX_JOBS 1024u

// One admitted request inside a launch.  Its rays own the global ids
// [begin, begin + count); every begin is a multiple of 32, so a 32-id chunk
// of the refilling engine never spans two requests.
struct ServeJob {
    const rq_bvh4_node* nodes4;
    const rq_triangle* tris;
    const uint32_t* perm;   // leaf order -> mesh triangle id
    const float* pos;       // mesh vertices (xyz, 12-B stride) for generated rays
    const uint32_t* idx;    // mesh indices
    const rq_ray* rays;     // RQ_RAYS_BUFFER
    rq_hit* hits;
    uint32_t* flag;         // host-mapped completion word: set to the launch's sequence number
    uint32_t begin, count, kind, seed;
    uint32_t ntri, flags, pad0, pad1;
};
static_assert(sizeof(ServeJob) == 96, "ServeJob layout");

// Launch one serving traversal over `njobs` jobs (device table `jobs`,
// device `begins` of njobs + 1 entries, the last = total ids).  `done`
// holds njobs zeroed counters; `ctr` one zeroed work counter.
int rq_launch_serve(rq_ctx* ctx, const ServeJob* jobs, const uint32_t* begins, uint32_t njobs, uint32_t total,
                    uint32_t max_depth4, uint32_t trace_flags, uint32_t seq, uint32_t* done, uint32_t* ctr,
                    cudaStream_t st);
int rq_launch_gen_mesh_rays(rq_ctx* ctx, const float* pos, const uint32_t* idx, uint32_t ntri, uint32_t kind,
                            uint32_t seed, uint32_t n, rq_ray* rays, uint32_t* any_flags, cudaStream_t st);
