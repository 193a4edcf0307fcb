// k_frame.cu — traversal kernels that generate their own rays.
//
//  k_gbuffer    one primary closest-hit ray per pixel
//               (benchmarks/exp1_visbuf/shaders/visbuf_raycast.comp:15-51,
//               optional per-pixel jitter), writing position, visibility
//               value, camera-facing face normal and t;
//  k_shadow_ao  per G-buffer pixel, the any-hit shadow rays of
//               shaders/tiled_lighting_ra.comp:223-253 and the cosine
//               hemisphere AO rays of shaders/rq_ao.comp:18-94, traced in the
//               same thread one after another — no ray or hit buffers touch
//               HBM.  Blocks are 16x8 pixel tiles, so a warp's rays toward one
//               light start side by side and walk the same nodes.
#include "rq_device.cuh"
#include "rq_internal.h"
#include "trace_core.cuh"

namespace {

constexpr int kTX = 16, kTY = 8, kT = kTX * kTY;

struct CamArgs {
    float m[16];
    float cx, cy, cz;
    uint32_t w, h, jitter, seed;
    float tmin, tmax;
};

// Per-pixel jitter draws in [0, 1].
__device__ __forceinline__ void jitter2(uint32_t seed, uint32_t pixel, float& jx, float& jy) {
    uint32_t h = rq::pcg_hash(seed ^ rq::pcg_hash(pixel));
    jx = __uint2float_rn(h) * RQ_INV_2POW32;
    jy = __uint2float_rn(rq::pcg_hash(h)) * RQ_INV_2POW32;
}

template <bool MT, int STACK>
__global__ void __launch_bounds__(kT) k_gbuffer(const rq_bvh4_node* __restrict__ nodes,
                                                const rq_triangle* __restrict__ tris,
                                                const uint32_t* __restrict__ perm, CamArgs c,
                                                rq_gbuffer_px* __restrict__ gbuf, uint32_t* err) {
    extern __shared__ int32_t s_stack[];
    const uint32_t px = blockIdx.x * kTX + threadIdx.x % kTX;
    const uint32_t py = blockIdx.y * kTY + threadIdx.x / kTX;
    if (px >= c.w || py >= c.h) return;
    const uint32_t pixel = py * c.w + px;
    float jx = 0.5f, jy = 0.5f;
    if (c.jitter) jitter2(c.seed, pixel, jx, jy);
    const float u = (__uint2float_rn(px) + jx) / __uint2float_rn(c.w);
    const float v = (__uint2float_rn(py) + jy) / __uint2float_rn(c.h);
    const float cl[4] = {u * 2.0f - 1.0f, v * 2.0f - 1.0f, 1.0f, 1.0f};
    float wt[4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
        wt[r] = ((c.m[r] * cl[0] + c.m[4 + r] * cl[1]) + c.m[8 + r] * cl[2]) + c.m[12 + r] * cl[3];
    const rq::F3 o{c.cx, c.cy, c.cz};
    const rq::F3 target{wt[0] / wt[3], wt[1] / wt[3], wt[2] / wt[3]};
    const rq::F3 d = rq::f3norm(rq::f3sub(target, o));
    rq::TraceResult res;
    rq::trace_ray<false, MT, false, STACK, kT>(nodes, tris, s_stack + threadIdx.x, o, d, c.tmin, c.tmax, res, err);
    float4* out = reinterpret_cast<float4*>(gbuf + pixel);
    if (res.idx == rq::kNoHit) {
        out[0] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
        out[1] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        return;
    }
    const rq::F3 p{o.x + res.t * d.x, o.y + res.t * d.y, o.z + res.t * d.z};
    const float4* tp = reinterpret_cast<const float4*>(tris + res.idx);
    const float4 a = rq::ldg4(tp), b = rq::ldg4(tp + 1), cc = rq::ldg4(tp + 2);
    const rq::F3 e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{cc.x - a.x, cc.y - a.y, cc.z - a.z};
    rq::F3 n = rq::f3norm(rq::f3cross(e1, e2));
    if (rq::f3dot(n, rq::f3sub(o, p)) < 0.0f) n = {-n.x, -n.y, -n.z};
    const uint32_t pid = perm ? __ldg(perm + res.idx) : res.idx;
    out[0] = make_float4(p.x, p.y, p.z, __uint_as_float(pid + 1u));
    out[1] = make_float4(n.x, n.y, n.z, res.t);
}

struct ShadeArgs {
    uint32_t w, h, nl, spp;
    float ao_tmax, ao_tmin, ao_bias, sh_tmin, sh_bias;
    float lx[RQ_MAX_LIGHTS], ly[RQ_MAX_LIGHTS], lz[RQ_MAX_LIGHTS], lr[RQ_MAX_LIGHTS];
};

// rq_ao.comp:27-45: rand() advances the hash state; cosine-weighted
// direction around N with the tangent frame of the shader.
__device__ __forceinline__ float ao_rand(uint32_t& seed) {
    seed = rq::ao_hash(seed);
    return __uint2float_rn(seed) * RQ_INV_2POW32;
}

__device__ __forceinline__ rq::F3 hemisphere(rq::F3 N, uint32_t& seed) {
    const float u1 = ao_rand(seed);
    const float u2 = ao_rand(seed);
    const float r = sqrtf(u1);
    const float theta = 6.2831853f * u2;
    float sn, cs;
    rq::sincos_taylor(theta, &sn, &cs);
    const float x = r * cs, y = r * sn, z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    const rq::F3 up = fabsf(N.z) < 0.999f ? rq::F3{0.0f, 0.0f, 1.0f} : rq::F3{1.0f, 0.0f, 0.0f};
    const rq::F3 tg = rq::f3norm(rq::f3cross(up, N));
    const rq::F3 bt = rq::f3cross(N, tg);
    return rq::f3norm(rq::F3{(tg.x * x + bt.x * y) + N.x * z, (tg.y * x + bt.y * y) + N.y * z,
                             (tg.z * x + bt.z * y) + N.z * z});
}

template <bool MT, bool STATS, int STACK>
__global__ void __launch_bounds__(kT) k_shadow_ao(const rq_bvh4_node* __restrict__ nodes,
                                                  const rq_triangle* __restrict__ tris,
                                                  const rq_gbuffer_px* __restrict__ gbuf, ShadeArgs s,
                                                  uint32_t* __restrict__ mask, float* __restrict__ ao,
                                                  unsigned long long* counters, uint32_t* err) {
    extern __shared__ int32_t s_stack[];
    const uint32_t px = blockIdx.x * kTX + threadIdx.x % kTX;
    const uint32_t py = blockIdx.y * kTY + threadIdx.x / kTX;
    const bool inside = px < s.w && py < s.h;
    uint32_t rays = 0, boxes = 0, ntris = 0;
    if (inside) {
        const uint32_t pixel = py * s.w + px;
        const float4* gp = reinterpret_cast<const float4*>(gbuf + pixel);
        const float4 g0 = __ldg(gp), g1 = __ldg(gp + 1);
        uint32_t m = 0;
        float occl = 1.0f;
        if (__float_as_uint(g0.w) != 0u) {
            const rq::F3 P{g0.x, g0.y, g0.z}, N{g1.x, g1.y, g1.z};
            rq::TraceResult res;
            const rq::F3 os{P.x + N.x * s.sh_bias, P.y + N.y * s.sh_bias, P.z + N.z * s.sh_bias};
            for (uint32_t k = 0; k < s.nl; ++k) {
                const rq::F3 tl{s.lx[k] - P.x, s.ly[k] - P.y, s.lz[k] - P.z};
                const float dist = sqrtf(rq::f3dot(tl, tl));
                if (dist > s.lr[k] || dist < 0.001f) continue;
                const rq::F3 L{tl.x / dist, tl.y / dist, tl.z / dist};
                if (fmaxf(0.0f, rq::f3dot(N, L)) <= 0.0f) continue;
                ++rays;
                rq::trace_ray<true, MT, STATS, STACK, kT>(nodes, tris, s_stack + threadIdx.x, os, L, s.sh_tmin,
                                                          dist - s.sh_bias, res, err);
                if (STATS) {
                    boxes += res.boxes;
                    ntris += res.tris;
                }
                if (res.idx == rq::kNoHit) m |= 1u << k;
            }
            if (s.spp) {
                uint32_t seed = pixel + 5544u;
                const rq::F3 oa{P.x + N.x * s.ao_bias, P.y + N.y * s.ao_bias, P.z + N.z * s.ao_bias};
                float unocc = 0.0f;
                for (uint32_t i = 0; i < s.spp; ++i) {
                    const rq::F3 dir = hemisphere(N, seed);
                    ++rays;
                    rq::trace_ray<true, MT, STATS, STACK, kT>(nodes, tris, s_stack + threadIdx.x, oa, dir, s.ao_tmin,
                                                              s.ao_tmax, res, err);
                    if (STATS) {
                        boxes += res.boxes;
                        ntris += res.tris;
                    }
                    if (res.idx == rq::kNoHit) unocc += 1.0f;
                }
                occl = unocc / __uint2float_rn(s.spp);
            }
        }
        mask[pixel] = m;
        ao[pixel] = occl;
    }
    if (counters) {
        const uint32_t wsum = __reduce_add_sync(0xffffffffu, rays);
        if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(counters, (unsigned long long)wsum);
        if (STATS) {
            const uint32_t bsum = __reduce_add_sync(0xffffffffu, boxes);
            const uint32_t tsum = __reduce_add_sync(0xffffffffu, ntris);
            if ((threadIdx.x & 31) == 0) {
                atomicAdd(counters + 1, (unsigned long long)bsum);
                atomicAdd(counters + 2, (unsigned long long)tsum);
            }
        }
    }
}

template <class F>
cudaError_t with_stack(uint32_t bound, F&& f) {
    if (bound <= 32) return f(std::integral_constant<int, 32>{});
    if (bound <= 64) return f(std::integral_constant<int, 64>{});
    return f(std::integral_constant<int, 128>{});
}

template <class K>
cudaError_t prep(K kern, int stack) {
    size_t smem = size_t(stack) * kT * sizeof(int32_t);
    if (smem > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    return cudaSuccess;
}

}  // namespace

int rq_launch_gbuffer(rq_ctx* ctx, const rq_bvh* bvh, const rq_camera& cam, rq_gbuffer_px* gbuf, cudaStream_t st) {
    CamArgs c;
    for (int i = 0; i < 16; ++i) c.m[i] = cam.inv_view_proj[i];
    c.cx = cam.cam_pos[0];
    c.cy = cam.cam_pos[1];
    c.cz = cam.cam_pos[2];
    c.w = cam.width;
    c.h = cam.height;
    c.jitter = cam.jitter;
    c.seed = cam.seed;
    c.tmin = cam.tmin;
    c.tmax = cam.tmax;
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const bool mt = cam.flags & RQ_TRI_MT;
    dim3 grid((cam.width + kTX - 1) / kTX, (cam.height + kTY - 1) / kTY);
    cudaError_t e = with_stack(bound, [&](auto S) {
        constexpr int STACK = decltype(S)::value;
        auto k = mt ? k_gbuffer<true, STACK> : k_gbuffer<false, STACK>;
        cudaError_t r = prep(k, STACK);
        if (r != cudaSuccess) return r;
        k<<<grid, kT, size_t(STACK) * kT * 4, st>>>(bvh->nodes4, bvh->tris, bvh->perm, c, gbuf, ctx->d_err);
        return cudaGetLastError();
    });
    return rq_cuda_status(ctx, e, "gbuffer launch");
}

int rq_launch_shadow_ao(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_shade_params& p,
                        uint32_t* mask, float* ao, unsigned long long* counter, cudaStream_t st) {
    ShadeArgs s;
    s.w = p.width;
    s.h = p.height;
    s.nl = p.num_lights;
    s.spp = p.ao_spp;
    s.ao_tmax = p.ao_tmax;
    s.ao_tmin = p.ao_tmin;
    s.ao_bias = p.ao_bias;
    s.sh_tmin = p.shadow_tmin;
    s.sh_bias = p.shadow_bias;
    for (int k = 0; k < RQ_MAX_LIGHTS; ++k) {
        const bool on = uint32_t(k) < p.num_lights;
        s.lx[k] = on ? p.lights[k].pos[0] : 0.0f;
        s.ly[k] = on ? p.lights[k].pos[1] : 0.0f;
        s.lz[k] = on ? p.lights[k].pos[2] : 0.0f;
        s.lr[k] = on ? p.lights[k].radius : 0.0f;
    }
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const bool mt = p.flags & RQ_TRI_MT;
    const bool stats = (p.flags & RQ_SHADE_COUNT_TESTS) && counter;
    dim3 grid((p.width + kTX - 1) / kTX, (p.height + kTY - 1) / kTY);
    cudaError_t e = with_stack(bound, [&](auto S) {
        constexpr int STACK = decltype(S)::value;
        auto k = mt ? (stats ? k_shadow_ao<true, true, STACK> : k_shadow_ao<true, false, STACK>)
                    : (stats ? k_shadow_ao<false, true, STACK> : k_shadow_ao<false, false, STACK>);
        cudaError_t r = prep(k, STACK);
        if (r != cudaSuccess) return r;
        k<<<grid, kT, size_t(STACK) * kT * 4, st>>>(bvh->nodes4, bvh->tris, gbuf, s, mask, ao, counter, ctx->d_err);
        return cudaGetLastError();
    });
    return rq_cuda_status(ctx, e, "shadow/AO launch");
}
