// k_serve.cu — the traversal launch of the serving loop and its ray makers.
//
//  k_serve         one persistent launch over the rays of many requests,
//                  each on its own resident BVH: the refilling engine of
//                  trace_engine.cuh draws 32-id chunks from one id space in
//                  which request j owns [begin_j, begin_j + count_j) (begins
//                  aligned to 32, requests ordered smallest first).  A lane
//                  maps its id to the request through a cached range or a
//                  binary search over the begins staged in shared memory,
//                  makes the ray (caller buffer, or generated from (seed, i)
//                  on the request's mesh), and writes the hit to the
//                  request's output.  Finished rays are counted per request
//                  with one atomic per group of lanes that finish together;
//                  the lane that completes a request publishes the launch's
//                  sequence number to the request's host-mapped flag, so the
//                  host sees each request finish while the launch runs on.
//  k_gen_mesh_rays the same generated rays, written out (for checking and for
//                  callers that want the rays themselves).
#include "rq_device.cuh"
#include "rq_internal.h"
#include "rq_serve_internal.h"
#include "trace_engine.cuh"

namespace {

constexpr int kST = 128;
// idle lanes of a warp get new rays once this many of 32 are idle (16: the
// frame's tuned threshold; equal or faster than 1 on the serving stream)
#ifndef RQ_SERVE_REFILL
#define RQ_SERVE_REFILL 16
#endif
constexpr int kServeRefill = RQ_SERVE_REFILL;

// Ray i of a generated request: up to eight draws pcg_hash(base + k) / 2^32
// with base = pcg_hash(seed ^ pcg_hash(i)).
__device__ __forceinline__ float draw(uint32_t base, uint32_t k) {
    return __uint2float_rn(rq::pcg_hash(base + k)) * RQ_INV_2POW32;
}

__device__ __forceinline__ rq::F3 vtx(const float* pos, uint32_t v) {
    return rq::F3{__ldg(pos + 3ull * v), __ldg(pos + 3ull * v + 1), __ldg(pos + 3ull * v + 2)};
}

// Returns the any-hit flag of the ray.
//  RQ_RAYS_CLOSEST: origin U[-1,1]^2 at z = 2, direction
//    normalise(U(-0.3,0.3), U(-0.3,0.3), -1), [0.01, 1000], closest hit.
//  RQ_RAYS_SHADOW / RQ_RAYS_AO: a point of a uniformly drawn triangle
//    (folded barycentrics), face normal N turned to +z;
//    shadow: toward a light uniform in [-1,1]^2 x [2,2.5], from P + 0.04 N,
//    [0.01, dist - 0.04] (shaders/tiled_lighting_ra.comp:118-148);
//    AO: cosine hemisphere about N from P + 0.03 N, [0.01, 0.5]
//    (shaders/rq_ao.comp:32-45, 77-86).
__device__ __forceinline__ bool gen_ray(uint32_t kind, uint32_t seed, uint32_t i, const float* pos,
                                        const uint32_t* idx, uint32_t ntri, rq::F3& o, rq::F3& d, float& tmin,
                                        float& tmax) {
    const uint32_t base = rq::pcg_hash(seed ^ rq::pcg_hash(i));
    if (kind == RQ_RAYS_CLOSEST) {
        o = rq::F3{-1.0f + 2.0f * draw(base, 0), -1.0f + 2.0f * draw(base, 1), 2.0f};
        d = rq::f3norm(rq::F3{-0.3f + 0.6f * draw(base, 2), -0.3f + 0.6f * draw(base, 3), -1.0f});
        tmin = 0.01f;
        tmax = 1000.0f;
        return false;
    }
    const uint32_t t = rq::pcg_hash(base + 7u) % ntri;
    const rq::F3 v0 = vtx(pos, __ldg(idx + 3ull * t)), v1 = vtx(pos, __ldg(idx + 3ull * t + 1)),
                 v2 = vtx(pos, __ldg(idx + 3ull * t + 2));
    float a = draw(base, 0), b = draw(base, 1);
    if (a + b > 1.0f) {
        a = 1.0f - a;
        b = 1.0f - b;
    }
    const rq::F3 e1 = rq::f3sub(v1, v0), e2 = rq::f3sub(v2, v0);
    const rq::F3 P{v0.x + (e1.x * a + e2.x * b), v0.y + (e1.y * a + e2.y * b), v0.z + (e1.z * a + e2.z * b)};
    rq::F3 N = rq::f3norm(rq::f3cross(e1, e2));
    if (N.z < 0.0f) N = rq::F3{-N.x, -N.y, -N.z};
    tmin = 0.01f;
    if (kind == RQ_RAYS_SHADOW) {
        const rq::F3 L{-1.0f + 2.0f * draw(base, 2), -1.0f + 2.0f * draw(base, 3), 2.0f + 0.5f * draw(base, 4)};
        const rq::F3 tl = rq::f3sub(L, P);
        const float dist = sqrtf(rq::f3dot(tl, tl));
        d = rq::F3{tl.x / dist, tl.y / dist, tl.z / dist};
        o = rq::F3{P.x + N.x * 0.04f, P.y + N.y * 0.04f, P.z + N.z * 0.04f};
        tmax = dist - 0.04f;
    } else {
        d = rq::cosine_hemisphere(N, draw(base, 2), draw(base, 3));
        o = rq::F3{P.x + N.x * 0.03f, P.y + N.y * 0.03f, P.z + N.z * 0.03f};
        tmax = 0.5f;
    }
    return true;
}

struct ServeSrc {
    static constexpr bool kMulti = true;
    static constexpr bool kRoundEnd = true;
    struct Meta {
        uint32_t job, local;
    };
    uint32_t total;
    uint32_t njobs;
    uint32_t seq;
    const ServeJob* jobs;
    const uint32_t* s_begin;  // shared: njobs + 1
    uint32_t* done;
    // per-lane cache of the last request's id range
    uint32_t cj = 0, cb = 1, ce = 0;

    __device__ uint32_t find(uint32_t id) {
        if (id >= cb && id < ce) return cj;
        uint32_t lo = 0, hi = njobs - 1;  // last j with begin_j <= id
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (s_begin[mid] <= id)
                lo = mid;
            else
                hi = mid - 1;
        }
        cj = lo;
        cb = s_begin[lo];
        ce = s_begin[lo + 1];
        return lo;
    }

    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) {
        const uint32_t j = find(id);
        const ServeJob* jb = jobs + j;
        const uint32_t local = id - cb;
        if (local >= __ldg(&jb->count)) return false;  // padding up to the next 32-id start
        m.job = j;
        m.local = local;
        r.nodes = jb->nodes4;
        r.tris = jb->tris;
        const uint32_t kind = __ldg(&jb->kind);
        if (kind == RQ_RAYS_BUFFER) {
            const float4* rp = reinterpret_cast<const float4*>(jb->rays + local);
            const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
            r.o = rq::F3{r0.x, r0.y, r0.z};
            r.d = rq::F3{r1.x, r1.y, r1.z};
            r.tmin = r0.w;
            r.tmax = r1.w;
            r.any = (__ldg(&jb->flags) & RQ_TRACE_ANY) != 0u;
        } else {
            r.any = gen_ray(kind, __ldg(&jb->seed), local, jb->pos, jb->idx, __ldg(&jb->ntri), r.o, r.d, r.tmin,
                            r.tmax);
        }
        return true;
    }

    __device__ void finish(uint32_t, const Meta& m, const rq::Ray&, const rq::Hit& h) const {
        const ServeJob* jb = jobs + m.job;
        uint4 out = make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
        if (h.hit) out = make_uint4(1u, __float_as_uint(h.t), 0u, __ldg(jb->perm + h.idx));
        reinterpret_cast<uint4*>(jb->hits)[m.local] = out;
    }

    __device__ void round_end(bool fin, const Meta& m) const {
        const uint32_t fm = __ballot_sync(rq::kFull, fin);
        if (!fin) return;
        __threadfence();  // this lane's hit store before the count that publishes it
        const uint32_t peers = __match_any_sync(fm, m.job);
        if ((threadIdx.x & 31u) != uint32_t(__ffs(peers) - 1)) return;
        const uint32_t c = __popc(peers);
        const ServeJob* jb = jobs + m.job;
        if (atomicAdd(done + m.job, c) + c == __ldg(&jb->count)) {
            __threadfence_system();
            *reinterpret_cast<volatile uint32_t*>(jb->flag) = seq;
        }
    }
};

// At most 72 registers per thread (7 blocks of 128 threads per SM), the
// budget that measured fastest for the frame's any-hit traversal.  `stack`
// rows of shared memory per thread (the deepest tree's bound, at most STACK).
template <bool MT, int STACK>
__global__ void __launch_bounds__(kST, 7) k_serve(const ServeJob* __restrict__ jobs, const uint32_t* __restrict__ begins,
                                               uint32_t njobs, uint32_t total, uint32_t seq, uint32_t* done,
                                               uint32_t* ctr, uint32_t* err, int stack) {
    extern __shared__ int32_t smem[];
    uint32_t* s_begin = reinterpret_cast<uint32_t*>(smem);
    for (uint32_t k = threadIdx.x; k <= njobs; k += kST) s_begin[k] = __ldg(begins + k);
    __syncthreads();
    int32_t* stk = smem + ((njobs + 1 + 3) & ~3u);
    ServeSrc src;
    src.total = total;
    src.njobs = njobs;
    src.seq = seq;
    src.jobs = jobs;
    src.s_begin = s_begin;
    src.done = done;
    rq::trace_persistent<rq::kAnyPerRay, MT, false, STACK, kST>(nullptr, nullptr, src, ctr, stk + threadIdx.x, err,
                                                                 stack, nullptr, kServeRefill);
}

__global__ void __launch_bounds__(256) k_gen_mesh_rays(const float* __restrict__ pos,
                                                       const uint32_t* __restrict__ idx, uint32_t ntri,
                                                       uint32_t kind, uint32_t seed, uint32_t n, rq_ray* rays,
                                                       uint32_t* any_flags) {
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    if (i >= n) return;
    rq::F3 o, d;
    float tmin, tmax;
    const bool any = gen_ray(kind, seed, i, pos, idx, ntri, o, d, tmin, tmax);
    float4* rp = reinterpret_cast<float4*>(rays + i);
    rp[0] = make_float4(o.x, o.y, o.z, tmin);
    rp[1] = make_float4(d.x, d.y, d.z, tmax);
    if (any_flags) any_flags[i] = any ? RQ_TRACE_ANY : RQ_TRACE_CLOSEST;
}

template <class F>
cudaError_t with_stack(uint32_t bound, F&& f) {
    if (bound <= 32) return f(std::integral_constant<int, 32>{});
    if (bound <= 64) return f(std::integral_constant<int, 64>{});
    return f(std::integral_constant<int, 128>{});
}

}  // namespace

int rq_launch_serve(rq_ctx* ctx, const ServeJob* jobs, const uint32_t* begins, uint32_t njobs, uint32_t total,
                    uint32_t max_depth4, uint32_t trace_flags, uint32_t seq, uint32_t* done, uint32_t* ctr,
                    cudaStream_t st) {
    if (njobs == 0 || njobs > RQ_SERVE_MAX_JOBS) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad job count");
    const uint32_t bound = 3u * (max_depth4 + 2u) + 1u;
    if (bound > 128u) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "4-wide tree deeper than 40 levels");
    const bool mt = trace_flags & RQ_TRI_MT;
    cudaError_t e = with_stack(bound, [&](auto S) {
        constexpr int STACK = decltype(S)::value;
        auto kern = mt ? k_serve<true, STACK> : k_serve<false, STACK>;
        const size_t smem = size_t((njobs + 1 + 3) & ~3u) * 4u + size_t(bound) * kST * 4u;  // bound <= STACK
        const size_t smem_max = size_t((RQ_SERVE_MAX_JOBS + 1 + 3) & ~3u) * 4u + size_t(STACK) * kST * 4u;
        cudaError_t r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem_max));
        int per_sm = 0;
        if (r == cudaSuccess) r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kST, smem);
        if (r != cudaSuccess) return r;
        uint32_t blocks = uint32_t(ctx->num_sms) * uint32_t(per_sm > 0 ? per_sm : 1);
        blocks = std::min(blocks, (total + kST - 1) / kST);
        kern<<<blocks, kST, smem, st>>>(jobs, begins, njobs, total, seq, done, ctr, ctx->d_err, int(bound));
        return cudaGetLastError();
    });
    return rq_cuda_status(ctx, e, "serve launch");
}

int rq_launch_gen_mesh_rays(rq_ctx* ctx, const float* pos, const uint32_t* idx, uint32_t ntri, uint32_t kind,
                            uint32_t seed, uint32_t n, rq_ray* rays, uint32_t* any_flags, cudaStream_t st) {
    if (n == 0) return RQ_OK;
    k_gen_mesh_rays<<<(n + 255) / 256, 256, 0, st>>>(pos, idx, ntri, kind, seed, n, rays, any_flags);
    return rq_cuda_status(ctx, cudaGetLastError(), "mesh ray generation");
}
