// k_batch.cu — many meshes per launch.
//
//  k_batch_build  one persistent launch builds every mesh of a batch: each
//                 thread block takes the next mesh from a size-ordered queue
//                 (largest first) and runs the whole LBVH pipeline on it with
//                 block barriers — centroids and bounds, Morton codes, a
//                 stable block-level LSD radix sort, Karras nodes, leaves and
//                 the atomic refit, the scan, the depth-first node writes and
//                 the greedy 4-wide collapse.  The per-element steps are those
//                 of build_core.cuh, so every mesh's bytes equal a separate
//                 rq_build of that mesh.  Each block owns a scratch slice sized
//                 for the batch's largest mesh.
//  k_batch_trace  one persistent traversal launch over rays of all meshes
//                 (trace_engine.cuh with per-ray BVH and per-ray any hit).
#include <algorithm>
#include <vector>

#include "build_core.cuh"
#include "rq_batch.h"
#include "rq_device.cuh"
#include "rq_internal.h"
#include "trace_engine.cuh"

namespace {

// Build blocks of BT threads (256, 512 or 1024: a tuned shape); the sort
// ranks kSortItems keys per thread per tile.
constexpr int kSortItems = 8;
constexpr uint32_t kMaxLevels = 120;

struct BlockScratch {
    float4* cent;
    uint32_t* keys[2];
    uint32_t* vals[2];
    int32_t *kl, *kr;
    uint32_t *klo, *khi, *par_in, *par_lf;
    float4 *box_in, *box_lf;
    uint32_t *refit_flag, *c, *a;
    uint32_t* q;
    int32_t *cand, *child_q;
    uint32_t *sz, *par, *tail;
    unsigned long long* acc;
};

__host__ __device__ size_t carve_block(uintptr_t base, uint32_t n, BlockScratch& s) {
    Carve c{base, 0};
    const size_t N = n ? n : 1;
    s.cent = c.take<float4>(N);
    s.keys[0] = c.take<uint32_t>(N);
    s.keys[1] = c.take<uint32_t>(N);
    s.vals[0] = c.take<uint32_t>(N);
    s.vals[1] = c.take<uint32_t>(N);
    s.kl = c.take<int32_t>(N);
    s.kr = c.take<int32_t>(N);
    s.klo = c.take<uint32_t>(N);
    s.khi = c.take<uint32_t>(N);
    s.par_in = c.take<uint32_t>(N);
    s.par_lf = c.take<uint32_t>(N);
    s.box_in = c.take<float4>(2 * N);
    s.box_lf = c.take<float4>(2 * N);
    s.refit_flag = c.take<uint32_t>(N);
    s.c = c.take<uint32_t>(N);
    s.a = c.take<uint32_t>(N);
    s.q = c.take<uint32_t>(N);
    s.cand = c.take<int32_t>(4 * N);
    s.child_q = c.take<int32_t>(4 * N);
    s.sz = c.take<uint32_t>(N);
    s.par = c.take<uint32_t>(N);
    s.acc = c.take<unsigned long long>(N);
    s.tail = c.take<uint32_t>(64);
    return (c.off + 255) & ~size_t(255);
}

struct BuildArgs {
    const float* pos;
    uint32_t sf;
    const uint32_t* idx;
    const rq_mesh_desc* meshes;
    const uint32_t* order;
    uint32_t num_meshes;
    uint32_t max_leaf;
    uint32_t* mesh_ctr;
    char* scratch;
    size_t scratch_stride;
    uint32_t scratch_n;
    rq_bvh2_node* nodes2;
    rq_triangle* tris;
    uint32_t* perm;
    uint32_t* skeys;
    rq_bvh4_node* nodes4;
    int32_t* map4;
    uint32_t* counts;  // 4 per mesh
    uint32_t* err;
};

// Block-wide exclusive scan of one value per thread; *total = sum.
template <int BT>
__device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    constexpr int kBW = BT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kBW ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kBW) s_warp[lane] = w;
    }
    __syncthreads();
    const uint32_t r = (warp ? s_warp[warp - 1] : 0u) + x - v;
    *total = s_warp[kBW - 1];
    __syncthreads();
    return r;
}

// Stable LSD radix sort of n (key, value) pairs by the low 30 key bits, four
// 8-bit passes between (keys[0], vals[0]) and (keys[1], vals[1]); the result
// ends in buffer 0.  Each pass: a digit histogram, then tiles of BT x 8 keys
// ranked per warp with match_any (peers in lane order) and scattered at
// digit base + running tile offset — the same stable order as the onesweep
// kernels of k_sort.cu.
template <int BT>
__device__ void block_sort(BlockScratch& s, uint32_t n, uint32_t* s_hist, uint32_t* s_off, uint32_t (*s_wcnt)[256],
                           uint32_t* s_warp) {
    constexpr int kBW = BT / 32, kBT = BT, kSortTile = BT * kSortItems;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int pass = 0; pass < 4; ++pass) {
        const uint32_t shift = 8u * pass;
        const uint32_t* kin = s.keys[pass & 1];
        const uint32_t* vin = s.vals[pass & 1];
        uint32_t* kout = s.keys[(pass & 1) ^ 1];
        uint32_t* vout = s.vals[(pass & 1) ^ 1];
        if (threadIdx.x < 256) s_hist[threadIdx.x] = 0;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += kBT) atomicAdd(&s_hist[(kin[i] >> shift) & 255u], 1u);
        __syncthreads();
        uint32_t tot;
        const uint32_t hv = threadIdx.x < 256 ? s_hist[threadIdx.x] : 0u;
        const uint32_t ex = block_scan<BT>(hv, s_warp, &tot);
        if (threadIdx.x < 256) s_off[threadIdx.x] = ex;
        __syncthreads();
        for (uint32_t base = 0; base < n; base += kSortTile) {
            for (int i = threadIdx.x; i < kBW * 256; i += kBT) (&s_wcnt[0][0])[i] = 0;
            __syncthreads();
            uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
            for (int j = 0; j < kSortItems; ++j) {
                const uint32_t i = base + warp * (32 * kSortItems) + j * 32 + lane;
                const bool valid = i < n;
                key[j] = valid ? kin[i] : 0u;
                val[j] = valid ? vin[i] : 0u;
                const uint32_t act = __ballot_sync(0xffffffffu, valid);
                rank[j] = 0;
                if (valid) {
                    const uint32_t d = (key[j] >> shift) & 255u;
                    const uint32_t peers = __match_any_sync(act, d);
                    const int leader = __ffs(peers) - 1;
                    const uint32_t below = __popc(peers & ((1u << lane) - 1u));
                    uint32_t b = 0;
                    if (lane == leader) {
                        b = s_wcnt[warp][d];
                        s_wcnt[warp][d] = b + __popc(peers);
                    }
                    b = __shfl_sync(peers, b, leader);
                    rank[j] = b + below;
                }
                __syncwarp();
            }
            __syncthreads();
            uint32_t tile_total = 0;
            if (threadIdx.x < 256) {
                uint32_t run = 0;
                for (int w = 0; w < kBW; ++w) {
                    const uint32_t cnt = s_wcnt[w][threadIdx.x];
                    s_wcnt[w][threadIdx.x] = run;
                    run += cnt;
                }
                tile_total = run;
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < kSortItems; ++j) {
                const uint32_t i = base + warp * (32 * kSortItems) + j * 32 + lane;
                if (i < n) {
                    const uint32_t d = (key[j] >> shift) & 255u;
                    const uint32_t pos = s_off[d] + s_wcnt[warp][d] + rank[j];
                    kout[pos] = key[j];
                    vout[pos] = val[j];
                }
            }
            __syncthreads();
            if (threadIdx.x < 256) s_off[threadIdx.x] += tile_total;
            __syncthreads();
        }
    }
}

// Exclusive scan of c[0..n) into a[0..n), tiles of BT x 8 with a carry.
template <int BT>
__device__ void block_scan_array(const uint32_t* c, uint32_t* a, uint32_t n, uint32_t* s_warp) {
    uint32_t carry = 0;
    for (uint32_t base = 0; base < n; base += BT * 8) {
        const uint32_t i0 = base + threadIdx.x * 8;
        uint32_t v[8], sum = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[k] = i0 + k < n ? c[i0 + k] : 0u;
            sum += v[k];
        }
        uint32_t tot;
        uint32_t run = carry + block_scan<BT>(sum, s_warp, &tot);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (i0 + k < n) a[i0 + k] = run;
            run += v[k];
        }
        carry += tot;
    }
    __syncthreads();
}

template <int BT>
__global__ void __launch_bounds__(BT) k_batch_build(BuildArgs A) {
    constexpr int kBT = BT, kBW = BT / 32;
    __shared__ uint32_t s_hist[256], s_off[256];
    __shared__ uint32_t s_wcnt[kBW][256];
    __shared__ uint32_t s_warp[32];
    __shared__ float s_red[6][kBW];
    __shared__ uint32_t s_lvl[kMaxLevels + 2];
    __shared__ uint32_t s_job;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    BlockScratch S;
    carve_block(reinterpret_cast<uintptr_t>(A.scratch + A.scratch_stride * blockIdx.x), A.scratch_n, S);

    for (;;) {
        if (threadIdx.x == 0) s_job = atomicAdd(A.mesh_ctr, 1u);
        __syncthreads();
        const uint32_t job = s_job;
        __syncthreads();
        if (job >= A.num_meshes) break;
        const uint32_t m = A.order[job];
        const rq_mesh_desc md = A.meshes[m];
        const uint32_t n = md.num_triangles;
        const float* pos = A.pos + size_t(md.vertex_offset) * A.sf;
        const uint32_t* idx = A.idx + 3ull * md.triangle_offset;
        const size_t toff = md.triangle_offset;
        rq_bvh2_node* out2 = A.nodes2 + 2 * toff;
        rq_triangle* tris = A.tris + toff;
        uint32_t* perm = A.perm + toff;
        uint32_t* skeys = A.skeys + toff;
        rq_bvh4_node* out4 = A.nodes4 + toff;
        int32_t* map4 = A.map4 + 4 * toff;
        uint32_t* counts = A.counts + 4 * size_t(m);

        // ---- centroids, bounds
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t t = threadIdx.x; t < n; t += kBT) {
            rq::F3 p0, p1, p2;
            rq::load_tri(pos, A.sf, idx, t, p0, p1, p2);
            const float4 c = rq::centroid(p0, p1, p2);
            S.cent[t] = c;
            mn[0] = fminf(mn[0], c.x);
            mn[1] = fminf(mn[1], c.y);
            mn[2] = fminf(mn[2], c.z);
            mx[0] = fmaxf(mx[0], c.x);
            mx[1] = fmaxf(mx[1], c.y);
            mx[2] = fmaxf(mx[2], c.z);
            if (t + 1 < n) S.refit_flag[t] = 0u;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
            }
        if (lane == 0)
            for (int k = 0; k < 3; ++k) {
                s_red[k][warp] = mn[k];
                s_red[3 + k][warp] = mx[k];
            }
        __syncthreads();
        float lo[3], hi[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = s_red[k][0];
            hi[k] = s_red[3 + k][0];
            for (int w = 1; w < kBW; ++w) {
                lo[k] = fminf(lo[k], s_red[k][w]);
                hi[k] = fmaxf(hi[k], s_red[3 + k][w]);
            }
        }
        const float scale = rq::morton_scale(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
        for (uint32_t t = threadIdx.x; t < n; t += kBT) {
            S.keys[0][t] = rq::morton30(S.cent[t], lo[0], lo[1], lo[2], scale);
            S.vals[0][t] = t;
        }
        __syncthreads();

        // ---- sort, hierarchy, leaves + refit
        block_sort<BT>(S, n, s_hist, s_off, s_wcnt, s_warp);
        for (uint32_t i = threadIdx.x; i + 1 < n; i += kBT)
            rq::karras_node(S.keys[0], int(n), int(i), S.kl, S.kr, S.klo, S.khi, S.par_in, S.par_lf);
        if (n == 1 && threadIdx.x == 0) S.par_lf[0] = rq::kNoParent;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < n; k += kBT) {
            rq::leaf_step(k, pos, A.sf, idx, A.max_leaf, S.keys[0], S.vals[0], S.klo, S.khi, S.par_in, S.par_lf,
                          S.box_lf, S.c, tris, perm, skeys);
            rq::refit_walk<true>(k, S.kl, S.kr, S.par_in, S.par_lf, S.box_in, S.box_lf, S.refit_flag, A.err);
        }
        __syncthreads();

        // ---- depth-first binary nodes
        block_scan_array<BT>(S.c, S.a, n, s_warp);
        for (uint32_t p = threadIdx.x; p < n; p += kBT) {
            const uint32_t cp = rq::emit_step(p, n, A.max_leaf, S.kr, S.klo, S.khi, S.par_in, S.par_lf, S.box_in,
                                              S.box_lf, S.c, S.a, out2);
            if (p == n - 1) {
                counts[0] = S.a[p] + cp;
                counts[3] = A.max_leaf;
            }
        }
        __syncthreads();

        // ---- 4-wide collapse
        rq::CollapseIO io;
        io.n2 = out2;
        io.q = S.q;
        io.cand = S.cand;
        io.child_q = S.child_q;
        io.sz = S.sz;
        io.par = S.par;
        io.acc = S.acc;
        io.tail = S.tail;
        io.out4 = out4;
        io.map4 = map4;
        uint32_t total = 0, depth = 0;
        auto sync = []() {
            __syncthreads();
            return true;
        };
        if (rq::collapse_levels<false, true, 0>(io, threadIdx.x, kBT, s_lvl, kMaxLevels, sync, A.err, &total, &depth) &&
            threadIdx.x == 0) {
            counts[1] = total;
            counts[2] = depth;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ trace
template <bool STATS>
struct BatchSrc {
    static constexpr bool kMulti = true;
    struct Meta {
        const uint32_t* perm;
    };
    uint32_t total;
    const rq_ray* rays;
    const uint32_t* ray_mesh;
    const uint32_t* ray_flags;
    uint32_t flags;
    const rq_mesh_desc* meshes;
    const rq_bvh4_node* nodes4;
    const rq_triangle* tris;
    const uint32_t* perm;
    rq_hit* hits;
    rq_ray_stats* stats;

    __device__ bool make(uint32_t id, rq::Ray& r, Meta& m) const {
        const float4* rp = reinterpret_cast<const float4*>(rays + id);
        const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
        const size_t toff = __ldg(&meshes[__ldg(ray_mesh + id)].triangle_offset);
        r.o = rq::F3{r0.x, r0.y, r0.z};
        r.d = rq::F3{r1.x, r1.y, r1.z};
        r.tmin = r0.w;
        r.tmax = r1.w;
        r.nodes = nodes4 + toff;
        r.tris = tris + toff;
        r.any = ((ray_flags ? __ldg(ray_flags + id) : flags) & RQ_TRACE_ANY) != 0u;
        m.perm = perm + toff;
        return true;
    }

    __device__ void finish(uint32_t id, const Meta& m, const rq::Ray&, const rq::Hit& h) const {
        uint4 out = make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
        if (h.hit) out = make_uint4(1u, __float_as_uint(h.t), 0u, __ldg(m.perm + h.idx));
        reinterpret_cast<uint4*>(hits)[id] = out;
        if (STATS) reinterpret_cast<uint4*>(stats)[id] = make_uint4(h.hit ? 1u : 0u, h.boxes, h.tris, 0u);
    }
};

// Traversal blocks of TT threads, ray ids taken CHUNK at a time, and (REGS)
// launch bounds that hold registers to REGS per thread: the tuned shapes.
// The stack has `stack` rows (runtime, from the batch's deepest tree); idle
// lanes are refilled once `refill_min` of a warp's lanes are idle.
template <bool MT, bool STATS, int TT, int CHUNK, int REGS>
__global__ void __launch_bounds__(TT, 65536 / (TT * (REGS ? REGS : 65536 / TT)))
    k_batch_trace(const __grid_constant__ BatchSrc<STATS> src, uint32_t* ctr, uint32_t* err, int stack,
                  int refill_min) {
    extern __shared__ int32_t s_stack[];
    rq::trace_persistent<rq::kAnyPerRay, MT, STATS, 128, TT, const BatchSrc<STATS>, CHUNK>(
        nullptr, nullptr, src, ctr, s_stack + threadIdx.x, err, stack, nullptr, refill_min);
}

template <int BT>
int build_occupancy() {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_build<BT>, BT, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return per_sm;
}

template <class F>
cudaError_t with_build_shape(uint32_t bt, F&& f) {
    if (bt == 256) return f(std::integral_constant<int, 256>{});
    if (bt == 1024) return f(std::integral_constant<int, 1024>{});
    return f(std::integral_constant<int, 512>{});
}

// Kernel of a traversal shape (only the default shape has the counting and
// reference-arithmetic variants).
template <bool MT, bool STATS>
const void* trace_kernel(uint32_t tt, uint32_t chunk, uint32_t regs) {
#define RQ_SHAPE(T, C, R) \
    if (tt == T && chunk == C && regs == R) return reinterpret_cast<const void*>(k_batch_trace<MT, STATS, T, C, R>);
#define RQ_SHAPES(T, C) RQ_SHAPE(T, C, 0) RQ_SHAPE(T, C, 64) RQ_SHAPE(T, C, 80)
    if constexpr (!MT && !STATS) {
        RQ_SHAPES(64, 32) RQ_SHAPES(64, 64) RQ_SHAPES(128, 64) RQ_SHAPES(256, 32) RQ_SHAPES(256, 64)
        RQ_SHAPE(128, 32, 64) RQ_SHAPE(128, 32, 80)
        // a budget of 72 registers: 7 blocks of 128 (14 of 64) threads per SM
        RQ_SHAPE(64, 32, 72) RQ_SHAPE(64, 64, 72) RQ_SHAPE(128, 32, 72) RQ_SHAPE(128, 64, 72)
    }
    RQ_SHAPE(128, 32, 0)
#undef RQ_SHAPES
#undef RQ_SHAPE
    return nullptr;
}

}  // namespace

size_t rq_batch_block_scratch(uint32_t max_tris) {
    BlockScratch s;
    return carve_block(0, max_tris, s);
}

int rq_batch_build_occupancy(uint32_t threads) {
    if (threads == 256) return build_occupancy<256>();
    if (threads == 1024) return build_occupancy<1024>();
    if (threads == 512) return build_occupancy<512>();
    return 0;
}

bool rq_batch_trace_shape_ok(uint32_t threads, uint32_t chunk, uint32_t regs) {
    return trace_kernel<false, false>(threads, chunk, regs) != nullptr;
}

int rq_launch_batch_build(rq_ctx* ctx, rq_batch* b, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                          cudaStream_t st) {
    BuildArgs a;
    a.pos = pos;
    a.sf = stride_bytes / 4;
    a.idx = idx;
    a.meshes = b->d_meshes;
    a.order = b->d_order;
    a.num_meshes = b->num_meshes;
    a.max_leaf = b->max_leaf;
    a.mesh_ctr = b->d_ctr;
    a.scratch = static_cast<char*>(b->scratch);
    a.scratch_stride = b->scratch_stride;
    a.scratch_n = b->max_tris;
    a.nodes2 = b->nodes2;
    a.tris = b->tris;
    a.perm = b->perm;
    a.skeys = b->skeys;
    a.nodes4 = b->nodes4;
    a.map4 = b->map4;
    a.counts = b->d_counts;
    a.err = ctx->d_err;
    const uint32_t blocks = std::min(b->tune.build_blocks, b->build_slices);
    cudaError_t e = cudaMemsetAsync(b->d_ctr, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = with_build_shape(b->tune.build_threads, [&](auto T) {
            constexpr int BT = decltype(T)::value;
            k_batch_build<BT><<<blocks, BT, 0, st>>>(a);
            return cudaGetLastError();
        });
    return rq_cuda_status(ctx, e, "batch build launch");
}

int rq_launch_batch_trace(rq_ctx* ctx, const rq_batch* b, const rq_ray* rays, const uint32_t* ray_mesh,
                          const uint32_t* ray_flags, uint32_t n, uint32_t flags, rq_hit* hits, rq_ray_stats* stats,
                          uint32_t* ctr, cudaStream_t st) {
    const uint32_t bound = 3u * (b->max_depth + 2u) + 1u;
    if (bound > 128u) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "4-wide tree deeper than 40 levels");
    const bool mt = flags & RQ_TRI_MT;
    // the counting and reference-arithmetic variants run in the default shape
    const bool tuned = !mt && !stats;
    const uint32_t tt = tuned ? b->tune.trace_threads : 128u;
    const uint32_t chunk = tuned ? b->tune.trace_chunk : 32u;
    const uint32_t regs = tuned ? b->tune.trace_reg_cap : 0u;
    int refill_min = int(tuned && b->tune.trace_refill_min ? b->tune.trace_refill_min : 1u);
    // stack rows: the bound, rounded up to a multiple of 4 (16-B rows)
    const int stack = int((std::max(bound, b->tune.stack_entries) + 3u) & ~3u);
    const void* kern = mt ? (stats ? trace_kernel<true, true>(tt, chunk, regs) : trace_kernel<true, false>(tt, chunk, regs))
                          : (stats ? trace_kernel<false, true>(tt, chunk, regs) : trace_kernel<false, false>(tt, chunk, regs));
    if (!kern) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "no traversal kernel for this shape");
    const size_t smem = size_t(stack) * tt * sizeof(int32_t);
    cudaError_t e = cudaMemsetAsync(ctr, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess && smem > 48 * 1024)
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    int per_sm = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, int(tt), smem);
    if (e == cudaSuccess) {
        if (b->tune.trace_blocks_per_sm && int(b->tune.trace_blocks_per_sm) < per_sm)
            per_sm = int(b->tune.trace_blocks_per_sm);
        uint32_t blocks = uint32_t(ctx->num_sms) * uint32_t(per_sm > 0 ? per_sm : 1);
        blocks = std::max(1u, std::min(blocks, (n + tt - 1) / tt));
        uint32_t* err = ctx->d_err;
        if (stats) {
            BatchSrc<true> src{n, rays, ray_mesh, ray_flags, flags, b->d_meshes, b->nodes4, b->tris, b->perm, hits,
                               stats};
            void* args[] = {&src, &ctr, &err, const_cast<int*>(&stack), &refill_min};
            e = cudaLaunchKernel(kern, dim3(blocks), dim3(tt), args, smem, st);
        } else {
            BatchSrc<false> src{n, rays, ray_mesh, ray_flags, flags, b->d_meshes, b->nodes4, b->tris, b->perm, hits,
                                nullptr};
            void* args[] = {&src, &ctr, &err, const_cast<int*>(&stack), &refill_min};
            e = cudaLaunchKernel(kern, dim3(blocks), dim3(tt), args, smem, st);
        }
    }
    return rq_cuda_status(ctx, e, "batch trace launch");
}
