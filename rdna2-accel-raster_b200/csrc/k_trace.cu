// k_trace.cu — ray traversal kernels.
//
//  k_trace4   the engine's 4-wide traversal (rq_trace): per-thread stack in
//             shared memory sized from the tree's depth (3*depth+1 entries
//             always suffice: each node visit pops one entry and pushes at
//             most four), 128-B nodes read as eight 16-B vector loads, inner
//             nodes and leaf children both pushed as entries.  Closest hit:
//             hit children sorted near-to-far (ties by slot) and pushed
//             far-first; any hit: pushed slot 3..0 and stop at the first
//             accepted triangle.  Watertight or Moller-Trumbore triangles.
//  k_trace_radv  the same rules over a RADV image (Box32 + triangle nodes).
//  k_ref4     software_bvh_bvh4.comp:96-195 as published (24-entry stack that
//             drops overflow, leaves tested inline far-to-near, RayStats).
//  k_ref2     software_bvh_lds.comp:86-175 as published (hitFound flag).
#include <atomic>
#include "rq_device.cuh"
#include "rq_internal.h"
#include "trace_engine.cuh"

namespace {

constexpr int kT = 128;
// rq_trace's engine: idle lanes are refilled once half the warp is idle, and
// 8 blocks of kT threads share an SM (64 registers).  Measured on B200 over
// 2^20 procedural rays, coherent and incoherent, at 968 / 99,458 / 999,698
// triangles: 8-18 % faster than refilling every idle lane at once with no
// register cap at five of the six points, equal at the sixth (968
// triangles, incoherent).
constexpr int kTraceRefill = 16;
constexpr int kTraceBlocksPerSm = 8;

__device__ __forceinline__ void store_miss(rq_hit* hits, uint32_t i) {
    reinterpret_cast<uint4*>(hits)[i] = make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
}

// Ray source of rq_trace: rays from a buffer, hits to a buffer.
template <bool STATS, bool BARY>
struct BufSrc {
    struct Meta {};
    uint32_t total;
    const rq_ray* rays;
    const uint32_t* perm;
    rq_hit* hits;
    float* bary;
    rq_ray_stats* stats;

    __device__ bool make(uint32_t id, rq::Ray& r, Meta&) const {
        const float4* rp = reinterpret_cast<const float4*>(rays + id);
        const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
        r.o = rq::F3{r0.x, r0.y, r0.z};
        r.d = rq::F3{r1.x, r1.y, r1.z};
        r.tmin = r0.w;
        r.tmax = r1.w;
        return true;
    }

    __device__ void finish(uint32_t id, const Meta&, const rq::Ray&, const rq::Hit& h) const {
        if (h.hit) {
            const uint32_t pid = perm ? __ldg(perm + h.idx) : h.idx;
            reinterpret_cast<uint4*>(hits)[id] = make_uint4(1u, __float_as_uint(h.t), 0u, pid);
        } else {
            store_miss(hits, id);
        }
        if (BARY) reinterpret_cast<float2*>(bary)[id] = h.hit ? make_float2(h.u, h.v) : make_float2(0.f, 0.f);
        if (STATS) reinterpret_cast<uint4*>(stats)[id] = make_uint4(h.hit ? 1u : 0u, h.boxes, h.tris, 0u);
    }
};

template <bool ANY, bool MT, bool STATS, bool BARY, int STACK>
__global__ void __launch_bounds__(kT, kTraceBlocksPerSm) k_trace4(const rq_bvh4_node* __restrict__ nodes,
                                               const rq_triangle* __restrict__ tris,
                                               const __grid_constant__ BufSrc<STATS, BARY> src,
                                               const uint32_t* __restrict__ counts, uint32_t* ctr, uint32_t* err) {
    extern __shared__ int32_t s_stack[];
    // the stack variant was picked from the host's copy of the depth; the
    // live depth (after an in-place rebuild) must still fit
    if (blockIdx.x == 0 && threadIdx.x == 0 && 3u * __ldg(counts + 2) + 1u > uint32_t(STACK))
        rq::set_err(err, RQ_DERR_STACK);
    rq::trace_persistent<ANY, MT, STATS, STACK, kT>(nodes, tris, src, ctr, s_stack + threadIdx.x, err, STACK, nullptr,
                                                    kTraceRefill);
}

template <bool ANY, bool MT, bool BARY>
__global__ void __launch_bounds__(kT) k_trace_radv(const uint8_t* __restrict__ img, const rq_ray* __restrict__ rays,
                                                   uint32_t n, rq_hit* __restrict__ hits, float* __restrict__ bary,
                                                   uint32_t* err) {
    constexpr int STACK = 64;
    __shared__ uint32_t s_stack[STACK * kT];
    const uint32_t i = blockIdx.x * kT + threadIdx.x;
    if (i >= n) return;
    uint32_t* stk = s_stack + threadIdx.x;
    const uint8_t* base = img + RQ_RADV_BVH_OFFSET;
    const float4* rp = reinterpret_cast<const float4*>(rays + i);
    float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    rq::F3 o{r0.x, r0.y, r0.z}, d{r1.x, r1.y, r1.z};
    const float tmin = r0.w;
    float best = r1.w;
    rq::SlabRay sr;
    sr.ix = rq::safe_inv(d.x);
    sr.iy = rq::safe_inv(d.y);
    sr.iz = rq::safe_inv(d.z);
    sr.ox = o.x * sr.ix;
    sr.oy = o.y * sr.iy;
    sr.oz = o.z * sr.iz;
    rq::WtRay w;
    if (!MT) w = rq::wt_setup(d);
    uint32_t hit_id = 0xffffffffu;
    bool found = false;
    float hu = 0.0f, hv = 0.0f;
    stk[0] = RQ_RADV_NODE_BOX32;
    int sp = 1;
    while (sp > 0) {
        const uint32_t id = stk[(--sp) * kT];
        const uint32_t type = id & 7u;
        const float4* np = reinterpret_cast<const float4*>(base + (size_t(id & ~7u) << 3));
        if (type == RQ_RADV_NODE_BOX32) {
            const uint4 ch = __ldg(reinterpret_cast<const uint4*>(np));
            float cf[24];
#pragma unroll
            for (int q = 0; q < 6; ++q) {
                float4 v = rq::ldg4(np + 1 + q);
                cf[4 * q] = v.x;
                cf[4 * q + 1] = v.y;
                cf[4 * q + 2] = v.z;
                cf[4 * q + 3] = v.w;
            }
            const uint32_t ac[4] = {ch.x, ch.y, ch.z, ch.w};
            uint32_t he[4];
            float ht[4];
            int nh = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (ac[k] == RQ_RADV_INVALID_NODE) continue;
                float tn;
                if (rq::slab(sr, tmin, best, cf[6 * k], cf[6 * k + 3], cf[6 * k + 1], cf[6 * k + 4], cf[6 * k + 2],
                             cf[6 * k + 5], tn)) {
                    int pos = nh;
                    if (!ANY) {
                        while (pos > 0 && ht[pos - 1] > tn) {
                            he[pos] = he[pos - 1];
                            ht[pos] = ht[pos - 1];
                            --pos;
                        }
                    }
                    he[pos] = ac[k];
                    ht[pos] = tn;
                    ++nh;
                }
            }
            if (sp + nh > STACK) {
                rq::set_err(err, RQ_DERR_STACK);
                nh = STACK - sp;
            }
            for (int j = nh - 1; j >= 0; --j) stk[(sp++) * kT] = he[j];
        } else if (type == RQ_RADV_NODE_TRIANGLE) {
            float4 a = rq::ldg4(np), b = rq::ldg4(np + 1), c = rq::ldg4(np + 2), dd = rq::ldg4(np + 3);
            rq::F3 v0{a.x, a.y, a.z}, v1{a.w, b.x, b.y}, v2{b.z, b.w, c.x};
            float t, u, v;
            bool ok = MT ? rq::mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v) : rq::wt_test(w, o, v0, v1, v2, t, u, v);
            if (ok && t >= tmin && t < best) {
                best = t;
                hit_id = __float_as_uint(dd.x);  // triangle_id at byte 48
                found = true;
                hu = u;
                hv = v;
                if (ANY) break;
            }
        }
    }
    if (found) {
        reinterpret_cast<uint4*>(hits)[i] = make_uint4(1u, __float_as_uint(best), 0u, hit_id);
    } else {
        store_miss(hits, i);
    }
    if (BARY) reinterpret_cast<float2*>(bary)[i] = found ? make_float2(hu, hv) : make_float2(0.f, 0.f);
}

__global__ void __launch_bounds__(kT) k_ref4(const rq_bvh4_node* __restrict__ nodes,
                                             const rq_triangle* __restrict__ tris, const rq_ray* __restrict__ rays,
                                             uint32_t n, rq_ray_stats* __restrict__ stats, rq_hit* __restrict__ hits) {
    __shared__ int32_t s_stack[24 * kT];
    const uint32_t idx = blockIdx.x * kT + threadIdx.x;
    if (idx >= n) return;
    int32_t* stk = s_stack + threadIdx.x;
    const rq_ray r = rays[idx];
    rq::F3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
    rq::F3 inv{fabsf(d.x) > 1e-6f ? 1.0f / d.x : 1e6f, fabsf(d.y) > 1e-6f ? 1.0f / d.y : 1e6f,
               fabsf(d.z) > 1e-6f ? 1.0f / d.z : 1e6f};
    const float tmin = r.tmin;
    float hitT = r.tmax;
    int hitPrim = -1;
    uint32_t boxTests = 0, triTests = 0;
    stk[0] = 0;
    int ptr = 1;
    while (ptr > 0) {
        const rq_bvh4_node nd = nodes[stk[(--ptr) * kT]];
        boxTests += 4;
        float tEntry[4], tExit[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float t0x = (nd.min_x[k] - o.x) * inv.x, t1x = (nd.max_x[k] - o.x) * inv.x;
            float t0y = (nd.min_y[k] - o.y) * inv.y, t1y = (nd.max_y[k] - o.y) * inv.y;
            float t0z = (nd.min_z[k] - o.z) * inv.z, t1z = (nd.max_z[k] - o.z) * inv.z;
            tEntry[k] = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), tmin));
            tExit[k] = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fminf(fmaxf(t0z, t1z), hitT));
        }
        int slot[4];
        float ht[4];
        int hc = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (nd.child_count[k] != 0 && tExit[k] >= tEntry[k]) {
                slot[hc] = k;
                ht[hc] = tEntry[k];
                ++hc;
            }
        if (hc == 0) continue;
        for (int a = 0; a < hc - 1; ++a)
            for (int b = a + 1; b < hc; ++b)
                if (ht[a] < ht[b]) {
                    float tt = ht[a];
                    ht[a] = ht[b];
                    ht[b] = tt;
                    int ts = slot[a];
                    slot[a] = slot[b];
                    slot[b] = ts;
                }
        for (int a = 0; a < hc; ++a) {
            int k = slot[a];
            if (nd.child_count[k] > 0) {
                uint32_t first = uint32_t(~nd.child_index[k]);
                uint32_t cnt = uint32_t(nd.child_count[k]);
                triTests += cnt;
                for (uint32_t p = 0; p < cnt; ++p) {
                    const rq_triangle tr = tris[first + p];
                    rq::F3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]},
                        v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                    float t, u, v;
                    if (!rq::mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v)) continue;
                    if (t >= tmin && t < hitT) {
                        hitT = t;
                        hitPrim = int(first + p);
                    }
                }
            } else if (nd.child_count[k] < 0) {
                if (ptr < 24) stk[(ptr++) * kT] = nd.child_index[k];
            }
        }
    }
    if (stats) reinterpret_cast<uint4*>(stats)[idx] = make_uint4(hitPrim >= 0 ? 1u : 0u, boxTests, triTests, 0u);
    if (hits) {
        if (hitPrim >= 0)
            reinterpret_cast<uint4*>(hits)[idx] = make_uint4(1u, __float_as_uint(hitT), 0u, uint32_t(hitPrim));
        else
            store_miss(hits, idx);
    }
}

__device__ __forceinline__ bool ref2_box(const rq_bvh2_node& nd, rq::F3 o, rq::F3 inv, float closestT, float& tb) {
    float t0x = (nd.aabb_min[0] - o.x) * inv.x, t1x = (nd.aabb_max[0] - o.x) * inv.x;
    float t0y = (nd.aabb_min[1] - o.y) * inv.y, t1y = (nd.aabb_max[1] - o.y) * inv.y;
    float t0z = (nd.aabb_min[2] - o.z) * inv.z, t1z = (nd.aabb_max[2] - o.z) * inv.z;
    float tNear = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fminf(t0z, t1z));
    float tFar = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
    tb = tNear;
    return (tFar >= fmaxf(0.0f, tNear)) && (tNear < closestT);
}

__device__ __forceinline__ float ref2_clamp(float x) { return fabsf(x) > 1e-8f ? x : (x >= 0.0f ? 1e-8f : -1e-8f); }

__global__ void __launch_bounds__(kT) k_ref2(const rq_bvh2_node* __restrict__ nodes,
                                             const rq_triangle* __restrict__ tris, const rq_ray* __restrict__ rays,
                                             uint32_t n, float t_eps, uint32_t* __restrict__ flags) {
    __shared__ uint32_t s_stack[32 * kT];
    const uint32_t idx = blockIdx.x * kT + threadIdx.x;
    if (idx >= n) return;
    uint32_t* stk = s_stack + threadIdx.x;
    const rq_ray r = rays[idx];
    rq::F3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
    rq::F3 inv{1.0f / ref2_clamp(d.x), 1.0f / ref2_clamp(d.y), 1.0f / ref2_clamp(d.z)};
    float closestT = r.tmax;
    uint32_t hitFound = 0;
    int sp = 0;
    stk[(sp++) * kT] = 0;
    while (sp > 0) {
        const rq_bvh2_node nd = nodes[stk[(--sp) * kT]];
        float tb;
        if (!ref2_box(nd, o, inv, closestT, tb)) continue;
        if (nd.left_child < 0) {
            uint32_t start = uint32_t(~nd.left_child);
            for (int32_t q = 0; q < nd.right_child; ++q) {
                const rq_triangle tr = tris[start + uint32_t(q)];
                rq::F3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]},
                    v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                float t, u, v;
                if (!rq::mt_test(o, d, v0, v1, v2, 1e-8f, t, u, v)) continue;
                if (t > t_eps && t < closestT) {
                    closestT = t;
                    hitFound = 1;
                }
            }
        } else {
            uint32_t l = uint32_t(nd.left_child), rr = uint32_t(nd.right_child);
            float tl, tr;
            bool hl = ref2_box(nodes[l], o, inv, closestT, tl), hr = ref2_box(nodes[rr], o, inv, closestT, tr);
            if (hl && hr) {
                if (tl < tr) {
                    if (sp < 32) stk[(sp++) * kT] = rr;
                    if (sp < 32) stk[(sp++) * kT] = l;
                } else {
                    if (sp < 32) stk[(sp++) * kT] = l;
                    if (sp < 32) stk[(sp++) * kT] = rr;
                }
            } else if (hl) {
                if (sp < 32) stk[(sp++) * kT] = l;
            } else if (hr) {
                if (sp < 32) stk[(sp++) * kT] = rr;
            }
        }
    }
    flags[idx] = hitFound;
}

template <bool ANY, bool MT, bool STATS, bool BARY, int STACK>
cudaError_t launch4(rq_ctx* ctx, const rq_bvh* b, const rq_ray* rays, uint32_t n, rq_hit* hits, float* bary,
                    rq_ray_stats* stats, cudaStream_t st) {
    auto kern = k_trace4<ANY, MT, STATS, BARY, STACK>;
    const size_t smem = size_t(STACK) * kT * sizeof(int32_t);
    // blocks per SM of this variant, found on its first launch on each device
    // (the shared-memory attribute is per device; the host calls cost more
    // than a small launch's kernel)
    static std::atomic<int> s_per_sm[64];
    const int dev = ctx->device;
    int per_sm = (dev >= 0 && dev < 64) ? s_per_sm[dev].load(std::memory_order_relaxed) : 0;
    cudaError_t e = cudaSuccess;
    if (per_sm == 0) {
        if (smem > 48 * 1024) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kT, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) per_sm = 1;
        if (dev >= 0 && dev < 64) s_per_sm[dev].store(per_sm, std::memory_order_relaxed);
    }
    // persistent grid: every SM filled, never more blocks than 32-ray chunks
    uint32_t blocks = uint32_t(ctx->num_sms) * uint32_t(per_sm > 0 ? per_sm : 1);
    const uint32_t need = (n + kT - 1) / kT;
    if (blocks > need) blocks = need;
    BufSrc<STATS, BARY> src;
    src.total = n;
    src.rays = rays;
    src.perm = b->perm;
    src.hits = hits;
    src.bary = bary;
    src.stats = stats;
    e = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    kern<<<blocks, kT, smem, st>>>(b->nodes4, b->tris, src, b->d_counts, ctx->d_ctr, ctx->d_err);
    return cudaGetLastError();
}

template <bool ANY, bool MT, bool STATS, bool BARY>
cudaError_t launch4_stack(uint32_t bound, rq_ctx* ctx, const rq_bvh* b, const rq_ray* rays, uint32_t n,
                          rq_hit* hits, float* bary, rq_ray_stats* stats, cudaStream_t st) {
    if (bound <= 32) return launch4<ANY, MT, STATS, BARY, 32>(ctx, b, rays, n, hits, bary, stats, st);
    if (bound <= 64) return launch4<ANY, MT, STATS, BARY, 64>(ctx, b, rays, n, hits, bary, stats, st);
    return launch4<ANY, MT, STATS, BARY, 128>(ctx, b, rays, n, hits, bary, stats, st);
}

template <bool ANY, bool MT>
cudaError_t launch4_opts(uint32_t bound, bool ex, rq_ctx* ctx, const rq_bvh* b, const rq_ray* rays, uint32_t n,
                         rq_hit* hits, float* bary, rq_ray_stats* stats, cudaStream_t st) {
    if (ex) return launch4_stack<ANY, MT, true, true>(bound, ctx, b, rays, n, hits, bary, stats, st);
    return launch4_stack<ANY, MT, false, false>(bound, ctx, b, rays, n, hits, bary, stats, st);
}

}  // namespace

int rq_launch_trace(rq_ctx* ctx, const rq_bvh* bvh, const rq_ray* rays, uint32_t n, uint32_t flags, rq_hit* hits,
                    float* bary, rq_ray_stats* stats, cudaStream_t st) {
    if (n == 0) return RQ_OK;
    // stack entries: 3 per level below the root plus one, with two levels of
    // headroom for in-place rebuilds whose depth the host has not seen yet
    uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    if (3u * bvh->h_counts[2] + 1u > 128u)
        return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "4-wide tree deeper than 42 levels");
    // With stats or barycentrics requested, the kernel variant that records
    // both is used; a null destination gets a scratch sink.
    rq_ray_stats* st_out = stats;
    float* ba_out = bary;
    if ((stats != nullptr) != (bary != nullptr)) {
        size_t need = size_t(n) * (stats ? 8 : 16);
        int rc = rq_ensure_scratch(ctx, need, st);
        if (rc) return rc;
        if (!stats) st_out = static_cast<rq_ray_stats*>(ctx->scratch);
        if (!bary) ba_out = static_cast<float*>(ctx->scratch);
    }
    const bool any = flags & RQ_TRACE_ANY, mt = flags & RQ_TRI_MT;
    const bool ex = stats || bary;
    cudaError_t e;
    if (any && mt)
        e = launch4_opts<true, true>(bound, ex, ctx, bvh, rays, n, hits, ba_out, st_out, st);
    else if (any)
        e = launch4_opts<true, false>(bound, ex, ctx, bvh, rays, n, hits, ba_out, st_out, st);
    else if (mt)
        e = launch4_opts<false, true>(bound, ex, ctx, bvh, rays, n, hits, ba_out, st_out, st);
    else
        e = launch4_opts<false, false>(bound, ex, ctx, bvh, rays, n, hits, ba_out, st_out, st);
    return rq_cuda_status(ctx, e, "trace launch");
}

int rq_launch_trace_ref4(rq_ctx* ctx, const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                         uint32_t n, rq_ray_stats* stats, rq_hit* hits, cudaStream_t st) {
    if (n == 0) return RQ_OK;
    k_ref4<<<(n + kT - 1) / kT, kT, 0, st>>>(nodes, tris, rays, n, stats, hits);
    return rq_cuda_status(ctx, cudaGetLastError(), "reference bvh4 trace launch");
}

int rq_launch_trace_ref2(rq_ctx* ctx, const rq_bvh2_node* nodes, const rq_triangle* tris, const rq_ray* rays,
                         uint32_t n, float t_eps, uint32_t* flags, cudaStream_t st) {
    if (n == 0) return RQ_OK;
    k_ref2<<<(n + kT - 1) / kT, kT, 0, st>>>(nodes, tris, rays, n, t_eps, flags);
    return rq_cuda_status(ctx, cudaGetLastError(), "reference bvh2 trace launch");
}

int rq_launch_trace_radv(rq_ctx* ctx, const void* img, uint64_t bytes, const rq_ray* rays, uint32_t n,
                         uint32_t flags, rq_hit* hits, float* bary, cudaStream_t st) {
    (void)bytes;
    if (n == 0) return RQ_OK;
    const uint8_t* im = static_cast<const uint8_t*>(img);
    const bool any = flags & RQ_TRACE_ANY, mt = flags & RQ_TRI_MT, b = bary != nullptr;
    dim3 g((n + kT - 1) / kT);
#define RQ_RADV_CASE(A, M, B) k_trace_radv<A, M, B><<<g, kT, 0, st>>>(im, rays, n, hits, bary, ctx->d_err)
    if (any && mt && b) RQ_RADV_CASE(true, true, true);
    else if (any && mt) RQ_RADV_CASE(true, true, false);
    else if (any && b) RQ_RADV_CASE(true, false, true);
    else if (any) RQ_RADV_CASE(true, false, false);
    else if (mt && b) RQ_RADV_CASE(false, true, true);
    else if (mt) RQ_RADV_CASE(false, true, false);
    else if (b) RQ_RADV_CASE(false, false, true);
    else RQ_RADV_CASE(false, false, false);
#undef RQ_RADV_CASE
    return rq_cuda_status(ctx, cudaGetLastError(), "radv trace launch");
}
