/*
 * rq_serve.h — serving form of the ray-query engine: a request loop that
 * takes (mesh, ray batch) queries as they arrive, keeps the meshes' BVHs
 * resident in device memory, admits requests against a memory budget, and
 * coalesces the rays of many requests into shared persistent traversal
 * launches that overlap on the device (continuous batching).
 *
 * The reference has no serving layer: its hosts build one BVH and dispatch
 * one trace per mesh (benchmarks/microbench/microbench_main.cpp:175-294,
 * src/main.cpp:871-873).  The plain mode of this server reproduces that
 * shape — one request, one launch, wait, next — and is the comparison point
 * for the batched mode.  Per-request results are the same in both modes and
 * the same as rq_build + rq_trace on the request's mesh and rays, bit for bit.
 *
 * Threading: rq_server_submit / rq_server_poll / rq_server_replay may be
 * called from any host thread; one worker thread per server owns the device
 * work.  The server creates its own rq_ctx and streams on `device`.
 */
#ifndef RQ_SERVE_H
#define RQ_SERVE_H

#include "rq.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rq_server rq_server;

/* Ray sources of a request.  The generated kinds draw their rays on the
 * device from (seed, ray index, mesh) inside the traversal launch, so no ray
 * buffer touches device memory; rq_gen_mesh_rays writes the same rays out. */
#define RQ_RAYS_BUFFER 0u   /* caller's device rays (rq_ray), flags from rq_request.flags */
#define RQ_RAYS_SHADOW 1u   /* any hit: surface point -> light in [-1,1]^2 x [2,2.5]
                               (shaders/tiled_lighting_ra.comp:118-148 offsets: +0.04 N, tmin 0.01, tmax dist-0.04) */
#define RQ_RAYS_AO 2u       /* any hit: cosine hemisphere about the face normal
                               (shaders/rq_ao.comp:32-94: +0.03 N, tmin 0.01, tmax 0.5) */
#define RQ_RAYS_CLOSEST 3u  /* closest hit: origin U[-1,1]^2 at z=2, dir normalise(U(-.3,.3), U(-.3,.3), -1) */

#define RQ_SERVE_BATCHED 0u /* coalesce admitted requests into shared launches, several in flight */
#define RQ_SERVE_PLAIN 1u   /* one request per launch, one launch in flight */

typedef struct rq_server_config {
    uint64_t hbm_budget_bytes;  /* resident meshes: vertices + indices + BVH arrays */
    uint32_t mode;              /* RQ_SERVE_BATCHED or RQ_SERVE_PLAIN */
    uint32_t slots;             /* traversal launches in flight, 1..8 (plain: 1) */
    uint32_t max_wave_rays;     /* rays coalesced into one launch (a request larger than this runs alone) */
    uint32_t max_wave_requests; /* requests coalesced into one launch, 1..1024 (plain: 1) */
    uint32_t max_leaf;          /* leaf size of the builds, 1..16 */
    uint32_t trace_flags;       /* 0 watertight, RQ_TRI_MT reference Moeller-Trumbore */
    uint32_t rebuild;           /* plain mode only: rebuild the mesh's BVH (in place) before every request,
                                   the per-request build + trace of the reference's hosts */
} rq_server_config;

typedef struct rq_request {
    uint32_t mesh;      /* id returned by rq_server_add_mesh */
    uint32_t kind;      /* RQ_RAYS_* */
    uint32_t num_rays;  /* >= 1 */
    uint32_t seed;      /* generated kinds */
    uint32_t flags;     /* RQ_RAYS_BUFFER: RQ_TRACE_ANY or RQ_TRACE_CLOSEST */
    uint32_t reserved;
    const rq_ray* rays; /* RQ_RAYS_BUFFER: num_rays device rays, valid until completion */
    rq_hit* hits;       /* num_rays device results (16-B aligned), written before completion */
    uint64_t user;      /* returned in the completion */
} rq_request;

typedef struct rq_completion {
    uint64_t ticket;
    uint64_t user;
    int32_t status;     /* RQ_OK, RQ_ERR_BUDGET (mesh larger than the budget), RQ_ERR_INVALID_ARG,
                           RQ_ERR_DEVICE_TIMEOUT / RQ_ERR_CUDA (the launch failed) */
    uint32_t built;     /* 1 when the request's mesh was uploaded and built for it */
    double t_submit;    /* seconds on rq_server_now's clock */
    double t_admit;     /* launch enqueued */
    double t_done;      /* worker saw the request's completion flag */
} rq_completion;

typedef struct rq_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t launches;       /* traversal launches */
    uint64_t builds, evictions;
    uint64_t rays;           /* rays of completed requests */
    uint64_t resident_bytes, peak_resident_bytes;
    uint64_t max_requests_per_launch;
    uint64_t max_launches_in_flight;
} rq_server_stats;

int rq_server_create(int device, const rq_server_config* cfg, rq_server** out);
/* Stops the worker after the requests already submitted complete. */
int rq_server_destroy(rq_server* s);
/* Register a mesh (host arrays are copied into pinned memory; uploaded and
 * built when a request first needs it, evicted least-recently-used when the
 * budget needs room).  Reserves the build scratch for it. */
int rq_server_add_mesh(rq_server* s, const float* pos, uint32_t num_vertices, const uint32_t* idx,
                       uint32_t num_triangles, uint32_t* mesh_id);
/* Device bytes a resident mesh of this size takes (vertices, indices, BVH). */
uint64_t rq_server_mesh_bytes(uint32_t num_vertices, uint32_t num_triangles);
int rq_server_submit(rq_server* s, const rq_request* req, uint64_t* ticket);
/* Submit reqs[i] at arrival[i] seconds after the call (sorted ascending);
 * returns when the last one is submitted.  tickets may be NULL. */
int rq_server_replay(rq_server* s, const rq_request* reqs, const double* arrival, uint32_t n, uint64_t* tickets);
/* Move up to `capacity` completions out of the server (completion order). */
int rq_server_poll(rq_server* s, rq_completion* out, uint32_t capacity, uint32_t* count);
/* Wait until every submitted request has completed (RQ_ERR_DEVICE_TIMEOUT
 * after timeout_ms). */
int rq_server_drain(rq_server* s, uint32_t timeout_ms);
double rq_server_now(const rq_server* s);
int rq_server_stats_get(rq_server* s, rq_server_stats* out);
const char* rq_server_last_error(const rq_server* s);
/* Cancel a submitted request: if it has not been admitted to a launch yet, it
 * completes with RQ_ERR_CANCELLED; otherwise it completes as it would have.
 * RQ_ERR_INVALID_ARG for a ticket this server never issued. */
int rq_server_cancel(rq_server* s, uint64_t ticket);

/* Host-side fault injection (for failure-handling tests): the next `count`
 * mesh uploads fail as if the device allocation had failed (their requests
 * complete with RQ_ERR_OOM), or the next `count` launches fail as if the
 * launch had returned an error (their requests complete with RQ_ERR_CUDA).
 * The server keeps serving afterwards.  Nothing faults on the device. */
#define RQ_FAULT_ALLOC 1u
#define RQ_FAULT_LAUNCH 2u
int rq_server_inject_fault(rq_server* s, uint32_t kind, uint32_t count);

/* The rays a generated request of `kind` traces (mesh-local primitive ids):
 * writes num_rays rays and, per ray, its trace flag (RQ_TRACE_ANY /
 * RQ_TRACE_CLOSEST) when any_flags is not NULL. */
int rq_gen_mesh_rays(rq_ctx* ctx, const float* pos, const uint32_t* idx, uint32_t num_triangles, uint32_t kind,
                     uint32_t seed, uint32_t num_rays, rq_ray* rays, uint32_t* any_flags, rq_stream stream);

#ifdef __cplusplus
}
#endif

#endif
