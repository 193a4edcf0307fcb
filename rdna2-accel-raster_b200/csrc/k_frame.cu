// k_frame.cu — traversal kernels that generate their own rays.
//
//  k_gbuffer_seq  one primary closest-hit ray per pixel and thread
//               (benchmarks/exp1_visbuf/shaders/visbuf_raycast.comp:15-51,
//               optional per-pixel jitter) -> position, visibility value,
//               camera-facing face normal, t.  Camera rays are coherent, so
//               the one-ray-per-thread schedule of trace_core.cuh wins.
//  k_shadow_ao  the any-hit shadow rays of shaders/tiled_lighting_ra.comp:
//               118-148 and the cosine-hemisphere AO rays of
//               shaders/rq_ao.comp:18-94, generated from the G-buffer inside
//               the kernel, on the refilling schedule of trace_engine.cuh
//               (a pixel's rays differ in length, so lanes must not wait for
//               one another).  A ray id names (8x4 pixel tile, ray kind k, pixel
//               in tile): the 32 ids of one chunk are the 32 pixels of a tile
//               casting toward the same light (or the same AO sample), the
//               most coherent batch a warp can trace.  A ray that reaches its
//               light / escapes sets bit k of its pixel's 64-bit result word
//               (lights in bits 0..31, AO samples in bits 32..63).
//  k_shade_finish  result words -> light mask and AO fraction per pixel.
//  k_reflect    the closest-hit reflection ray of
//               shaders/tiled_lighting_ra.comp:91-113 per G-buffer pixel,
//               on the refilling schedule (reflections off a rough surface
//               scatter), writing one hit record per pixel.
//  k_ao_depth   the AO rays of shaders/rq_ao.comp:47-97 from a depth buffer:
//               surface position and normal reconstructed from the pixel's
//               and its right and upper neighbours' depths, then the
//               cosine-hemisphere any-hit rays; k_ao_depth_finish turns the
//               per-pixel result bits into the AO fraction.
// No ray buffer touches HBM.
#include "rq_device.cuh"
#include "rq_internal.h"
#include "trace_core.cuh"
#include "trace_engine.cuh"

namespace {

constexpr int kT = 128;
constexpr uint32_t kTileW = 8, kTileH = 4;

struct CamArgs {
    float m[16];
    float cx, cy, cz;
    uint32_t w, h, jitter, seed;
    float tmin, tmax;
};

__device__ __forceinline__ bool tile_pixel(uint32_t tile, uint32_t j, uint32_t tiles_x, uint32_t w, uint32_t h,
                                           uint32_t& pixel) {
    const uint32_t px = (tile % tiles_x) * kTileW + (j & 7u);
    const uint32_t py = (tile / tiles_x) * kTileH + (j >> 3);
    if (px >= w || py >= h) return false;
    pixel = py * w + px;
    return true;
}

// Per-pixel jitter draws in [0, 1].
__device__ __forceinline__ void jitter2(uint32_t seed, uint32_t pixel, float& jx, float& jy) {
    uint32_t h = rq::pcg_hash(seed ^ rq::pcg_hash(pixel));
    jx = __uint2float_rn(h) * RQ_INV_2POW32;
    jy = __uint2float_rn(rq::pcg_hash(h)) * RQ_INV_2POW32;
}

struct GbufSrc {
    struct Meta {
        uint32_t pixel;
    };
    uint32_t total;
    uint32_t tiles_x;
    CamArgs c;
    const rq_triangle* tris;
    const uint32_t* perm;
    rq_gbuffer_px* gbuf;

    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) const {
        uint32_t pixel;
        if (!tile_pixel(id >> 5, id & 31u, tiles_x, c.w, c.h, pixel)) return false;
        m.pixel = pixel;
        const uint32_t px = pixel % c.w, py = pixel / c.w;
        float jx = 0.5f, jy = 0.5f;
        if (c.jitter) jitter2(c.seed, pixel, jx, jy);
        const float u = (__uint2float_rn(px) + jx) / __uint2float_rn(c.w);
        const float v = (__uint2float_rn(py) + jy) / __uint2float_rn(c.h);
        const float cl[4] = {u * 2.0f - 1.0f, v * 2.0f - 1.0f, 1.0f, 1.0f};
        float wt[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            wt[k] = ((c.m[k] * cl[0] + c.m[4 + k] * cl[1]) + c.m[8 + k] * cl[2]) + c.m[12 + k] * cl[3];
        r.o = rq::F3{c.cx, c.cy, c.cz};
        const rq::F3 target{wt[0] / wt[3], wt[1] / wt[3], wt[2] / wt[3]};
        r.d = rq::f3norm(rq::f3sub(target, r.o));
        r.tmin = c.tmin;
        r.tmax = c.tmax;
        return true;
    }

    __device__ void finish(uint32_t, const Meta& m, const rq::Ray& r, const rq::Hit& h) const {
        float4* out = reinterpret_cast<float4*>(gbuf + m.pixel);
        if (!h.hit) {
            out[0] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
            out[1] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
            return;
        }
        const rq::F3 p{r.o.x + h.t * r.d.x, r.o.y + h.t * r.d.y, r.o.z + h.t * r.d.z};
        const float4* tp = reinterpret_cast<const float4*>(tris + h.idx);
        const float4 a = rq::ldg4(tp), b = rq::ldg4(tp + 1), cc = rq::ldg4(tp + 2);
        const rq::F3 e1{b.x - a.x, b.y - a.y, b.z - a.z}, e2{cc.x - a.x, cc.y - a.y, cc.z - a.z};
        rq::F3 n = rq::f3norm(rq::f3cross(e1, e2));
        if (rq::f3dot(n, rq::f3sub(r.o, p)) < 0.0f) n = {-n.x, -n.y, -n.z};
        const uint32_t pid = perm ? __ldg(perm + h.idx) : h.idx;
        out[0] = make_float4(p.x, p.y, p.z, __uint_as_float(pid + 1u));
        out[1] = make_float4(n.x, n.y, n.z, h.t);
    }
};

struct ShadeArgs {
    uint32_t w, h, nl, spp;
    float ao_tmax, ao_tmin, ao_bias, sh_tmin, sh_bias;
    float lx[RQ_MAX_LIGHTS], ly[RQ_MAX_LIGHTS], lz[RQ_MAX_LIGHTS], lr[RQ_MAX_LIGHTS];
};

__device__ __forceinline__ float ao_rand(uint32_t& seed) {
    seed = rq::ao_hash(seed);
    return __uint2float_rn(seed) * RQ_INV_2POW32;
}

// rq_ao.comp:32-45 for sample s of the pixel: the hash state advances two
// draws per sample from y*W + x + 5544.
__device__ __forceinline__ rq::F3 hemisphere(rq::F3 N, uint32_t pixel, uint32_t s) {
    uint32_t seed = pixel + 5544u;
    for (uint32_t i = 0; i < 2 * s; ++i) seed = rq::ao_hash(seed);
    const float u1 = ao_rand(seed);
    const float u2 = ao_rand(seed);
    return rq::cosine_hemisphere(N, u1, u2);
}

template <bool STATS>
struct ShadeSrc {
    struct Meta {
        uint32_t pixel, bit;
    };
    uint32_t total;
    uint32_t tiles_x;
    uint32_t kinds;  // lights + AO samples
    const ShadeArgs* s;
    const rq_gbuffer_px* gbuf;
    unsigned long long* words;
    uint32_t rays = 0, boxes = 0, tris = 0;

    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) {
        const uint32_t q = id >> 5, k = q % kinds;
        uint32_t pixel;
        if (!tile_pixel(q / kinds, id & 31u, tiles_x, s->w, s->h, pixel)) return false;
        const float4* gp = reinterpret_cast<const float4*>(gbuf + pixel);
        const float4 g0 = __ldg(gp);
        if (__float_as_uint(g0.w) == 0u) return false;
        const float4 g1 = __ldg(gp + 1);
        const rq::F3 P{g0.x, g0.y, g0.z}, N{g1.x, g1.y, g1.z};
        m.pixel = pixel;
        m.bit = k;
        if (k < s->nl) {
            const rq::F3 tl{s->lx[k] - P.x, s->ly[k] - P.y, s->lz[k] - P.z};
            const float dist = sqrtf(rq::f3dot(tl, tl));
            if (dist > s->lr[k] || dist < 0.001f) return false;
            const rq::F3 L{tl.x / dist, tl.y / dist, tl.z / dist};
            if (fmaxf(0.0f, rq::f3dot(N, L)) <= 0.0f) return false;
            r.o = rq::F3{P.x + N.x * s->sh_bias, P.y + N.y * s->sh_bias, P.z + N.z * s->sh_bias};
            r.d = L;
            r.tmin = s->sh_tmin;
            r.tmax = dist - s->sh_bias;
        } else {
            m.bit = 32u + (k - s->nl);
            r.o = rq::F3{P.x + N.x * s->ao_bias, P.y + N.y * s->ao_bias, P.z + N.z * s->ao_bias};
            r.d = hemisphere(N, pixel, k - s->nl);
            r.tmin = s->ao_tmin;
            r.tmax = s->ao_tmax;
        }
        ++rays;
        return true;
    }

    __device__ void finish(uint32_t, const Meta& m, const rq::Ray&, const rq::Hit& h) {
        if (STATS) {
            boxes += h.boxes;
            tris += h.tris;
        }
        if (!h.hit) atomicOr(words + m.pixel, 1ull << m.bit);
    }
};

// One camera ray per thread, 16x8 pixels per block: primary rays are
// coherent, so lanes stay together without refilling.  `stack` rows of
// shared memory per thread (the tree's bound, at most STACK).
template <bool MT, int STACK>
__global__ void __launch_bounds__(kT) k_gbuffer_seq(const rq_bvh4_node* __restrict__ nodes,
                                                    const rq_triangle* __restrict__ tris,
                                                    const __grid_constant__ GbufSrc src, uint32_t* err, int stack) {
    extern __shared__ int32_t s_stack[];
    // each warp takes an 8x4 pixel tile of the block's 16x8 (the most compact
    // footprint, so its rays stay close)
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint32_t px = blockIdx.x * 16 + (w & 1u) * 8 + (l & 7u);
    const uint32_t py = blockIdx.y * 8 + (w >> 1) * 4 + (l >> 3);
    if (px >= src.c.w || py >= src.c.h) return;
    const uint32_t id = ((py / kTileH) * src.tiles_x + px / kTileW) * 32u + (py % kTileH) * kTileW + px % kTileW;
    rq::Ray r;
    GbufSrc::Meta m;
    src.make(id, r, m);
    rq::TraceResult res;
    rq::trace_ray<false, MT, false, STACK, kT>(nodes, tris, s_stack + threadIdx.x, r.o, r.d, r.tmin, r.tmax, res,
                                               err, stack);
    rq::Hit h;
    h.hit = res.idx != rq::kNoHit;
    h.t = res.t;
    h.idx = res.idx;
    h.u = res.u;
    h.v = res.v;
    h.boxes = res.boxes;
    h.tris = res.tris;
    src.finish(id, m, r, h);
}

// Camera rays on the refilling engine with in-loop refill (closest hit):
// rays that need few nodes hand their lane to the next pixel instead of
// waiting for the warp's longest ray.
template <bool MT, int TT, int REGS>
__global__ void __launch_bounds__(TT, 65536 / (TT * REGS))
    k_gbuffer_eng(const rq_bvh4_node* __restrict__ nodes, const rq_triangle* __restrict__ tris,
                  const __grid_constant__ GbufSrc src0, uint32_t* ctr, uint32_t* err, int stack, int refill_min,
                  int leaf_batch) {
    extern __shared__ __align__(16) int32_t s_stack[];
    GbufSrc src = src0;
    rq::trace_persistent<0, MT, false, 128, TT, GbufSrc, 32, 0, false, true>(
        nodes, tris, src, ctr, s_stack + threadIdx.x, err, stack, nullptr, refill_min, leaf_batch);
}

// TT threads per block, CHUNK ray ids per refill, REGS: launch bounds that
// hold registers to REGS (0: none) — the tuned shapes; `stack` rows per lane;
// idle lanes are refilled once `refill_min` of a warp's lanes are idle.
// INLOOP: rays finish and lanes refill inside the node loop (leaf_batch
// parked leaves end it).
template <bool MT, bool STATS, int TT, int CHUNK, int REGS, int TOP, bool SPEC, bool INLOOP = false>
__global__ void __launch_bounds__(TT, 65536 / (TT * (REGS ? REGS : 65536 / TT)))
    k_shadow_ao(const rq_bvh4_node* __restrict__ nodes, const rq_triangle* __restrict__ tris,
                const rq_gbuffer_px* __restrict__ gbuf, const __grid_constant__ ShadeArgs sa,
                unsigned long long* words, unsigned long long* counters, uint32_t* ctr, uint32_t* err, int stack,
                int refill_min, int leaf_batch) {
    extern __shared__ __align__(16) int32_t s_stack[];
    // shared memory: the stack (stack rows x TT), then the staged top levels
    float4* s_top = reinterpret_cast<float4*>(s_stack + stack * TT);
    if (TOP > 0) rq::stage_top<TOP>(nodes, s_top);
    ShadeSrc<STATS> src;
    src.kinds = sa.nl + sa.spp;
    src.tiles_x = (sa.w + kTileW - 1) / kTileW;
    src.total = src.tiles_x * ((sa.h + kTileH - 1) / kTileH) * src.kinds * 32u;
    src.s = &sa;
    src.gbuf = gbuf;
    src.words = words;
    rq::trace_persistent<1, MT, STATS, 128, TT, ShadeSrc<STATS>, CHUNK, TOP, SPEC, INLOOP>(
        nodes, tris, src, ctr, s_stack + threadIdx.x, err, stack, s_top, refill_min, leaf_batch);
    if (counters) {
        const uint32_t r = __reduce_add_sync(rq::kFull, src.rays);
        if ((threadIdx.x & 31u) == 0 && r) atomicAdd(counters, (unsigned long long)r);
        if (STATS) {
            const uint32_t b = __reduce_add_sync(rq::kFull, src.boxes);
            const uint32_t t = __reduce_add_sync(rq::kFull, src.tris);
            if ((threadIdx.x & 31u) == 0) {
                atomicAdd(counters + 1, (unsigned long long)b);
                atomicAdd(counters + 2, (unsigned long long)t);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_shade_finish(const rq_gbuffer_px* __restrict__ gbuf,
                                                      const unsigned long long* __restrict__ words, uint32_t npix,
                                                      uint32_t spp, uint32_t* __restrict__ mask,
                                                      float* __restrict__ ao) {
    const uint32_t p = blockIdx.x * 256 + threadIdx.x;
    if (p >= npix) return;
    const unsigned long long w = words[p];
    const bool vis = reinterpret_cast<const uint4*>(gbuf + p)->w != 0u;
    mask[p] = uint32_t(w);
    ao[p] = (vis && spp) ? __uint2float_rn(uint32_t(__popcll(w >> 32))) / __uint2float_rn(spp) : 1.0f;
}

// ------------------------------------------------------------- reflection
struct ReflSrc {
    struct Meta {
        uint32_t pixel;
    };
    uint32_t total;
    uint32_t tiles_x;
    uint32_t w, h;
    float cx, cy, cz, tmin, tmax, bias;
    const rq_gbuffer_px* gbuf;
    const uint32_t* perm;
    rq_hit* hits;

    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) const {
        uint32_t pixel;
        if (!tile_pixel(id >> 5, id & 31u, tiles_x, w, h, pixel)) return false;
        const float4* gp = reinterpret_cast<const float4*>(gbuf + pixel);
        const float4 g0 = __ldg(gp);
        if (__float_as_uint(g0.w) == 0u) {  // no surface: the shader casts nothing
            reinterpret_cast<uint4*>(hits)[pixel] = make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
            return false;
        }
        const float4 g1 = __ldg(gp + 1);
        const rq::F3 P{g0.x, g0.y, g0.z}, N{g1.x, g1.y, g1.z};
        const rq::F3 V = rq::f3norm(rq::f3sub(P, rq::F3{cx, cy, cz}));
        const float k = 2.0f * rq::f3dot(N, V);  // reflect(V, N) = V - 2 dot(N, V) N
        r.d = rq::F3{V.x - k * N.x, V.y - k * N.y, V.z - k * N.z};
        r.o = rq::F3{P.x + N.x * bias, P.y + N.y * bias, P.z + N.z * bias};
        r.tmin = tmin;
        r.tmax = tmax;
        m.pixel = pixel;
        return true;
    }

    __device__ void finish(uint32_t, const Meta& m, const rq::Ray&, const rq::Hit& h) const {
        const uint4 rec = h.hit ? make_uint4(1u, __float_as_uint(h.t), 0u, perm ? __ldg(perm + h.idx) : h.idx)
                                : make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
        reinterpret_cast<uint4*>(hits)[m.pixel] = rec;
    }
};

template <bool MT, int TT, int REGS>
__global__ void __launch_bounds__(TT, 65536 / (TT * REGS))
    k_reflect(const rq_bvh4_node* __restrict__ nodes, const rq_triangle* __restrict__ tris,
              const __grid_constant__ ReflSrc src0, uint32_t* ctr, uint32_t* err, int stack) {
    extern __shared__ __align__(16) int32_t s_stack[];
    ReflSrc src = src0;
    rq::trace_persistent<0, MT, false, 128, TT, ReflSrc>(nodes, tris, src, ctr, s_stack + threadIdx.x, err, stack);
}

// ------------------------------------------------------------ AO from depth
struct AoDepthArgs {
    float m[16];
    float cx, cy, cz;
    uint32_t w, h, spp;  // spp >= 1
    float maxd, tmin, bias;
};

// inv_view_proj * (u*2-1, v*2-1, d, 1), divided by w.
__device__ __forceinline__ rq::F3 unproject(const float* m, float u, float v, float d) {
    const float n[4] = {u * 2.0f - 1.0f, v * 2.0f - 1.0f, d, 1.0f};
    float o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = ((m[k] * n[0] + m[4 + k] * n[1]) + m[8 + k] * n[2]) + m[12 + k] * n[3];
    return rq::F3{o[0] / o[3], o[1] / o[3], o[2] / o[3]};
}

// rq_ao.comp:51-68: position from the depth at the pixel centre, normal from
// the right and upper neighbours (depth clamped at the edge), turned toward
// the camera.  False where depth >= 1.
__device__ __forceinline__ bool depth_surface(const AoDepthArgs& a, const float* __restrict__ depth, uint32_t px,
                                              uint32_t py, rq::F3& P, rq::F3& N) {
    const float d = __ldg(depth + size_t(py) * a.w + px);
    if (d >= 1.0f) return false;
    const float fw = __uint2float_rn(a.w), fh = __uint2float_rn(a.h);
    const float u = (__uint2float_rn(px) + 0.5f) / fw, v = (__uint2float_rn(py) + 0.5f) / fh;
    const float tx = 1.0f / fw, ty = 1.0f / fh;
    const float dr = __ldg(depth + size_t(py) * a.w + (px + 1 < a.w ? px + 1 : a.w - 1));
    const float du = __ldg(depth + size_t(py + 1 < a.h ? py + 1 : a.h - 1) * a.w + px);
    P = unproject(a.m, u, v, d);
    const rq::F3 pr = unproject(a.m, u + tx, v, dr);
    const rq::F3 pu = unproject(a.m, u, v + ty, du);
    N = rq::f3norm(rq::f3cross(rq::f3sub(pr, P), rq::f3sub(pu, P)));
    if (rq::f3dot(N, rq::f3sub(rq::F3{a.cx, a.cy, a.cz}, P)) < 0.0f) N = {-N.x, -N.y, -N.z};
    return true;
}

struct AoDepthSrc {
    struct Meta {
        uint32_t pixel, bit;
    };
    uint32_t total;
    uint32_t tiles_x;
    const AoDepthArgs* a;
    const float* depth;
    uint32_t* words;
    uint32_t rays = 0;

    // id = ((tile * spp + sample) << 5) | pixel in the 8x4 tile
    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) {
        const uint32_t q = id >> 5, k = q % a->spp;
        uint32_t pixel;
        if (!tile_pixel(q / a->spp, id & 31u, tiles_x, a->w, a->h, pixel)) return false;
        rq::F3 P, N;
        if (!depth_surface(*a, depth, pixel % a->w, pixel / a->w, P, N)) return false;
        m.pixel = pixel;
        m.bit = k;
        r.o = rq::F3{P.x + N.x * a->bias, P.y + N.y * a->bias, P.z + N.z * a->bias};
        r.d = hemisphere(N, pixel, k);
        r.tmin = a->tmin;
        r.tmax = a->maxd;
        ++rays;
        return true;
    }

    __device__ void finish(uint32_t, const Meta& m, const rq::Ray&, const rq::Hit& h) {
        if (!h.hit) atomicOr(words + m.pixel, 1u << m.bit);
    }
};

template <bool MT, int TT, int REGS>
__global__ void __launch_bounds__(TT, 65536 / (TT * REGS))
    k_ao_depth(const rq_bvh4_node* __restrict__ nodes, const rq_triangle* __restrict__ tris,
               const float* __restrict__ depth, const __grid_constant__ AoDepthArgs a, uint32_t* words,
               unsigned long long* counters, uint32_t* ctr, uint32_t* err, int stack) {
    extern __shared__ __align__(16) int32_t s_stack[];
    AoDepthSrc src;
    src.tiles_x = (a.w + kTileW - 1) / kTileW;
    src.total = src.tiles_x * ((a.h + kTileH - 1) / kTileH) * a.spp * 32u;
    src.a = &a;
    src.depth = depth;
    src.words = words;
    rq::trace_persistent<1, MT, false, 128, TT, AoDepthSrc>(nodes, tris, src, ctr, s_stack + threadIdx.x, err, stack);
    if (counters) {
        const uint32_t r = __reduce_add_sync(rq::kFull, src.rays);
        if ((threadIdx.x & 31u) == 0 && r) atomicAdd(counters, (unsigned long long)r);
    }
}

__global__ void __launch_bounds__(256) k_ao_depth_finish(const float* __restrict__ depth,
                                                         const uint32_t* __restrict__ words, uint32_t npix,
                                                         uint32_t spp, float* __restrict__ ao) {
    const uint32_t p = blockIdx.x * 256 + threadIdx.x;
    if (p >= npix) return;
    ao[p] = __ldg(depth + p) >= 1.0f ? 1.0f : __uint2float_rn(uint32_t(__popc(words[p]))) / __uint2float_rn(spp);
}

// Grid of a persistent traversal kernel: every SM filled to its occupancy.
cudaError_t persistent_grid(rq_ctx* ctx, const void* k, int threads, size_t smem, uint32_t& blocks) {
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem);
    blocks = uint32_t(ctx->num_sms) * uint32_t(per_sm > 0 ? per_sm : 1);
    return e;
}

template <class F>
cudaError_t with_stack(uint32_t bound, F&& f) {
    if (bound <= 32) return f(std::integral_constant<int, 32>{});
    if (bound <= 64) return f(std::integral_constant<int, 64>{});
    return f(std::integral_constant<int, 128>{});
}

// Shadow/AO kernel of a launch shape (only the default shape has the
// counting and reference-arithmetic variants).
template <bool MT, bool STATS>
const void* shade_kernel(const rq_trace_tuning& t) {
#define RQ_SHAPE(T, C, R, L, S)                                                                             \
    if (t.threads == T && t.chunk == C && t.reg_cap == R && t.top_levels == L && (t.speculative != 0) == S) \
        return reinterpret_cast<const void*>(k_shadow_ao<MT, STATS, T, C, R, L, S>);
#define RQ_SHAPES(T, C)                                                                              \
    RQ_SHAPE(T, C, 0, 0, false) RQ_SHAPE(T, C, 64, 0, false) RQ_SHAPE(T, C, 80, 0, false) RQ_SHAPE(T, C, 80, 4, false) \
    RQ_SHAPE(T, C, 80, 0, true)
    if constexpr (!MT && !STATS) {
        RQ_SHAPES(64, 32) RQ_SHAPES(64, 64) RQ_SHAPES(128, 64) RQ_SHAPES(256, 32) RQ_SHAPES(256, 64)
        RQ_SHAPE(128, 32, 64, 0, false) RQ_SHAPE(128, 32, 80, 0, false) RQ_SHAPE(128, 32, 80, 4, false)
        RQ_SHAPE(128, 32, 80, 0, true)
        // a budget of 72 registers: 7 blocks of 128 (14 of 64) threads per SM
        RQ_SHAPE(64, 32, 72, 0, false) RQ_SHAPE(64, 32, 72, 0, true) RQ_SHAPE(64, 64, 72, 0, false)
        RQ_SHAPE(64, 64, 72, 0, true) RQ_SHAPE(128, 32, 72, 0, false) RQ_SHAPE(128, 32, 72, 0, true)
        RQ_SHAPE(128, 64, 72, 0, false) RQ_SHAPE(128, 64, 72, 0, true)
        RQ_SHAPE(64, 64, 64, 0, true) RQ_SHAPE(128, 64, 64, 0, true) RQ_SHAPE(256, 64, 64, 0, true)
    }
    RQ_SHAPE(128, 32, 0, 0, false)
#undef RQ_SHAPES
#undef RQ_SHAPE
    return nullptr;
}

// Shapes with in-loop refill (speculative, leaf_batch > 0).
template <bool MT, bool STATS>
const void* shade_kernel_inloop(const rq_trace_tuning& t) {
#define RQ_SHAPE(T, C, R)                                                                      \
    if (t.threads == T && t.chunk == C && t.reg_cap == R && t.top_levels == 0 && t.speculative) \
        return reinterpret_cast<const void*>(k_shadow_ao<MT, STATS, T, C, R, 0, true, true>);
    if constexpr (!MT && !STATS) {
        RQ_SHAPE(64, 32, 64) RQ_SHAPE(64, 64, 64) RQ_SHAPE(128, 32, 64) RQ_SHAPE(128, 64, 64) RQ_SHAPE(256, 32, 64)
        RQ_SHAPE(256, 64, 64) RQ_SHAPE(128, 64, 72) RQ_SHAPE(256, 64, 72)
    }
#undef RQ_SHAPE
    return nullptr;
}

template <bool MT, bool STATS>
const void* shade_kernel_any(const rq_trace_tuning& t) {
    return t.leaf_batch ? shade_kernel_inloop<MT, STATS>(t) : shade_kernel<MT, STATS>(t);
}

}  // namespace

bool rq_shade_shape_ok(const rq_trace_tuning& t) { return shade_kernel_any<false, false>(t) != nullptr; }

int rq_launch_gbuffer(rq_ctx* ctx, const rq_bvh* bvh, const rq_camera& cam, rq_gbuffer_px* gbuf, cudaStream_t st) {
    GbufSrc src;
    CamArgs& c = src.c;
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
    src.tiles_x = (cam.width + kTileW - 1) / kTileW;
    src.total = src.tiles_x * ((cam.height + kTileH - 1) / kTileH) * 32u;
    src.tris = bvh->tris;
    src.perm = bvh->perm;
    src.gbuf = gbuf;
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const bool mt = cam.flags & RQ_TRI_MT;
    if (ctx->camera.engine) {
        constexpr int kET = 128, kER = 64;
        const int stack = int((bound + 3u) & ~3u);
        const void* k = mt ? reinterpret_cast<const void*>(k_gbuffer_eng<true, kET, kER>)
                           : reinterpret_cast<const void*>(k_gbuffer_eng<false, kET, kER>);
        const size_t smem = size_t(stack) * kET * sizeof(int32_t);
        uint32_t blocks = 0;
        cudaError_t e = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(uint32_t), st);
        if (e == cudaSuccess) e = persistent_grid(ctx, k, kET, smem, blocks);
        if (e == cudaSuccess) {
            const rq_bvh4_node* nodes = bvh->nodes4;
            const rq_triangle* tris = bvh->tris;
            uint32_t* ctr = ctx->d_ctr;
            uint32_t* err = ctx->d_err;
            int stk = stack, rm = int(ctx->camera.refill_min), lb = int(ctx->camera.leaf_batch);
            void* args[] = {&nodes, &tris, &src, &ctr, &err, &stk, &rm, &lb};
            e = cudaLaunchKernel(k, dim3(blocks), dim3(kET), args, smem, st);
        }
        return rq_cuda_status(ctx, e, "gbuffer launch");
    }
    dim3 grid((cam.width + 15) / 16, (cam.height + 7) / 8);
    cudaError_t e = with_stack(bound, [&](auto S) {
        constexpr int STACK = decltype(S)::value;
        auto k = mt ? k_gbuffer_seq<true, STACK> : k_gbuffer_seq<false, STACK>;
        const size_t smem = size_t(bound) * kT * 4;  // bound <= STACK
        if (smem > 48 * 1024) {
            cudaError_t r = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
            if (r != cudaSuccess) return r;
        }
        k<<<grid, kT, smem, st>>>(bvh->nodes4, bvh->tris, src, ctx->d_err, int(bound));
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
    const uint32_t npix = p.width * p.height;
    int rc = rq_ensure_scratch(ctx, sizeof(unsigned long long) * size_t(npix) + 256, st);
    if (rc) return rc;
    unsigned long long* words = static_cast<unsigned long long*>(ctx->scratch);
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const bool mt = p.flags & RQ_TRI_MT;
    const bool stats = (p.flags & RQ_SHADE_COUNT_TESTS) && counter;
    uint32_t* ctr = ctx->d_ctr;
    cudaError_t e = cudaMemsetAsync(words, 0, sizeof(unsigned long long) * size_t(npix), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess && p.num_lights + p.ao_spp > 0) {
        // the counting and reference-arithmetic variants run in the default shape
        const rq_trace_tuning shape = (mt || stats) ? rq_trace_tuning{128, 32, 0, 0, 0, 1, 0} : ctx->shade_shape;
        const size_t top_bytes = shape.top_levels == 4 ? rq::TopLevels<4>::kBytes : 0;
        const void* k = mt ? (stats ? shade_kernel_any<true, true>(shape) : shade_kernel_any<true, false>(shape))
                           : (stats ? shade_kernel_any<false, true>(shape) : shade_kernel_any<false, false>(shape));
        if (!k) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no traversal kernel for this shape");
        // stack rows: the bound for the tree's depth, rounded up to 4
        const int stack = int((bound + 3u) & ~3u);
        const size_t smem = size_t(stack) * shape.threads * sizeof(int32_t) + top_bytes;
        if (smem > 48 * 1024) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        int per_sm = 0;
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, int(shape.threads), smem);
        if (e == cudaSuccess) {
            const uint32_t blocks = uint32_t(ctx->num_sms) * uint32_t(per_sm > 0 ? per_sm : 1);
            const rq_bvh4_node* nodes = bvh->nodes4;
            const rq_triangle* tris = bvh->tris;
            uint32_t* err = ctx->d_err;
            int refill_min = int(shape.refill_min ? shape.refill_min : 1u);
            int leaf_batch = int(shape.leaf_batch ? shape.leaf_batch : 32u);
            void* args[] = {&nodes, &tris, &gbuf, &s, &words, &counter, &ctr, &err, const_cast<int*>(&stack),
                            &refill_min, &leaf_batch};
            e = cudaLaunchKernel(k, dim3(blocks), dim3(shape.threads), args, smem, st);
        }
    }
    if (e == cudaSuccess) {
        k_shade_finish<<<(npix + 255) / 256, 256, 0, st>>>(gbuf, words, npix, p.ao_spp, mask, ao);
        e = cudaGetLastError();
    }
    return rq_cuda_status(ctx, e, "shadow/AO launch");
}

// Launch shapes of the reflection and depth-AO traversals: 128-thread
// blocks held to 64 registers (8 blocks, 32 warps per SM).
constexpr int kReflThreads = 128, kReflRegs = 64;
constexpr int kAoThreads = 128, kAoRegs = 64;

int rq_launch_reflect(rq_ctx* ctx, const rq_bvh* bvh, const rq_gbuffer_px* gbuf, const rq_reflect_params& p,
                      rq_hit* hits, cudaStream_t st) {
    ReflSrc src;
    src.w = p.width;
    src.h = p.height;
    src.tiles_x = (p.width + kTileW - 1) / kTileW;
    src.total = src.tiles_x * ((p.height + kTileH - 1) / kTileH) * 32u;
    src.cx = p.cam_pos[0];
    src.cy = p.cam_pos[1];
    src.cz = p.cam_pos[2];
    src.tmin = p.tmin;
    src.tmax = p.tmax;
    src.bias = p.bias;
    src.gbuf = gbuf;
    src.perm = bvh->perm;
    src.hits = hits;
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const int stack = int((bound + 3u) & ~3u);
    const bool mt = p.flags & RQ_TRI_MT;
    const void* k = mt ? reinterpret_cast<const void*>(k_reflect<true, kReflThreads, kReflRegs>)
                       : reinterpret_cast<const void*>(k_reflect<false, kReflThreads, kReflRegs>);
    const size_t smem = size_t(stack) * kReflThreads * sizeof(int32_t);
    uint32_t blocks = 0;
    cudaError_t e = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) e = persistent_grid(ctx, k, kReflThreads, smem, blocks);
    if (e == cudaSuccess) {
        const rq_bvh4_node* nodes = bvh->nodes4;
        const rq_triangle* tris = bvh->tris;
        uint32_t* ctr = ctx->d_ctr;
        uint32_t* err = ctx->d_err;
        int stk = stack;
        void* args[] = {&nodes, &tris, &src, &ctr, &err, &stk};
        e = cudaLaunchKernel(k, dim3(blocks), dim3(kReflThreads), args, smem, st);
    }
    return rq_cuda_status(ctx, e, "reflection launch");
}

int rq_launch_ao_depth(rq_ctx* ctx, const rq_bvh* bvh, const float* depth, const rq_ao_depth_params& p, float* ao,
                       unsigned long long* counters, cudaStream_t st) {
    AoDepthArgs a;
    for (int i = 0; i < 16; ++i) a.m[i] = p.inv_view_proj[i];
    a.cx = p.cam_pos[0];
    a.cy = p.cam_pos[1];
    a.cz = p.cam_pos[2];
    a.w = p.width;
    a.h = p.height;
    a.spp = p.spp > 1u ? p.spp : 1u;  // rq_ao.comp:71: max(1u, samplesPerPixel)
    a.maxd = p.max_distance;
    a.tmin = p.tmin;
    a.bias = p.bias;
    const uint32_t npix = p.width * p.height;
    int rc = rq_ensure_scratch(ctx, sizeof(uint32_t) * size_t(npix) + 256, st);
    if (rc) return rc;
    uint32_t* words = static_cast<uint32_t*>(ctx->scratch);
    const uint32_t bound = 3u * (bvh->h_counts[2] + 2u) + 1u;
    const int stack = int((bound + 3u) & ~3u);
    const bool mt = p.flags & RQ_TRI_MT;
    const void* k = mt ? reinterpret_cast<const void*>(k_ao_depth<true, kAoThreads, kAoRegs>)
                       : reinterpret_cast<const void*>(k_ao_depth<false, kAoThreads, kAoRegs>);
    const size_t smem = size_t(stack) * kAoThreads * sizeof(int32_t);
    uint32_t blocks = 0;
    cudaError_t e = cudaMemsetAsync(words, 0, sizeof(uint32_t) * size_t(npix), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_ctr, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) e = persistent_grid(ctx, k, kAoThreads, smem, blocks);
    if (e == cudaSuccess) {
        const rq_bvh4_node* nodes = bvh->nodes4;
        const rq_triangle* tris = bvh->tris;
        uint32_t* ctr = ctx->d_ctr;
        uint32_t* err = ctx->d_err;
        int stk = stack;
        void* args[] = {&nodes, &tris, &depth, &a, &words, &counters, &ctr, &err, &stk};
        e = cudaLaunchKernel(k, dim3(blocks), dim3(kAoThreads), args, smem, st);
    }
    if (e == cudaSuccess) {
        k_ao_depth_finish<<<(npix + 255) / 256, 256, 0, st>>>(depth, words, npix, a.spp, ao);
        e = cudaGetLastError();
    }
    return rq_cuda_status(ctx, e, "depth AO launch");
}
