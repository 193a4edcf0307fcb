// k_batch.cu — many meshes per launch.
//
//  k_batch_build  one persistent launch builds every mesh of a batch: a
//                 team takes the next mesh from a size-ordered queue (largest
//                 first) and runs the whole LBVH pipeline on it — centroids
//                 and bounds, Morton codes, a stable LSD radix sort, Karras
//                 nodes, leaves and the atomic refit, the scan, the
//                 depth-first node writes and the greedy 4-wide collapse.  A
//                 team is one block (block barriers) or, for the largest
//                 meshes, a thread-block cluster of 2 or 4 blocks meeting at
//                 cluster barriers and exchanging its sort histograms, scan
//                 totals and bounds through distributed shared memory, so
//                 that one large mesh no longer holds one SM for the whole
//                 launch.  The per-element steps are those of build_core.cuh,
//                 so every mesh's bytes equal a separate rq_build of that
//                 mesh.  Each block owns a scratch slice sized for the batch's
//                 largest mesh (a cluster works in its first block's).
//  k_batch_trace  one persistent traversal launch over rays of all meshes
//                 (trace_engine.cuh with per-ray BVH and per-ray any hit).
#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "build_core.cuh"
#include "rq_batch.h"
#include "rq_device.cuh"
#include "rq_internal.h"
#include "trace_engine.cuh"

namespace {

namespace cg = cooperative_groups;

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
    const uint32_t* order;  // largest mesh first
    uint32_t num_meshes;
    uint32_t num_big;       // order[0, num_big): built by clusters
    uint32_t max_leaf;
    uint32_t* mesh_ctr;     // [0] cluster queue, [1] single-block queue
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

// Shared memory of one build block.
template <int BT>
struct BuildSmem {
    uint32_t hist[256], off[256];
    uint32_t wcnt[BT / 32][256];
    uint32_t warp[32];
    float red[6][BT / 32];
    float bnd[6];    // the block's centroid bounds (min xyz, max xyz)
    uint32_t tot;    // the block's share of a scan
    uint32_t lvl[kMaxLevels + 2];
    uint32_t job;    // this block's mesh
    uint32_t cjob;   // the cluster's mesh (read from the cluster's first block)
};

// The C blocks that build one mesh: a thread-block cluster (C > 1) whose
// blocks meet at cluster barriers (release / acquire at cluster scope, so
// the scratch writes of one block are visible to the others after it) and
// read each other's partial sums through distributed shared memory, or one
// block (C == 1, block barriers).
template <int C>
struct Team {
    uint32_t rank;  // block rank in the cluster
    __device__ static void sync() {
        if constexpr (C == 1)
            __syncthreads();
        else
            cg::this_cluster().sync();
    }
    // p (a shared-memory address) in block r of the cluster
    template <class T>
    __device__ static const T* at(T* p, uint32_t r) {
        if constexpr (C == 1)
            return p;
        else
            return cg::this_cluster().map_shared_rank(p, r);
    }
};

// The tiles [beg, end) of n items (tiles of `tile`) that rank `rank` of C
// handles: contiguous ranges in rank order, so a stable pass over the ranks
// in turn is stable over the whole range.
__device__ __forceinline__ void rank_range(uint32_t n, uint32_t tile, uint32_t c, uint32_t rank, uint32_t& beg,
                                           uint32_t& end) {
    const uint32_t tiles = (n + tile - 1) / tile, per = (tiles + c - 1) / c;
    beg = min(min(rank * per, tiles) * tile, n);
    end = min(beg + per * tile, n);
}

// Stable LSD radix sort of n (key, value) pairs by the low 30 key bits, four
// 8-bit passes between (keys[0], vals[0]) and (keys[1], vals[1]); the result
// ends in buffer 0.  Each pass: a digit histogram per block over its range,
// every block's digit offsets from all blocks' histograms (the digit's
// global base plus the counts of the lower ranks), then tiles of BT x 8 keys
// ranked per warp with match_any (peers in lane order) and scattered at
// digit offset + running tile offset — the same stable order as the
// onesweep kernels of k_sort.cu.
template <int BT, int C>
__device__ void team_sort(Team<C> tm, BlockScratch& s, uint32_t n, BuildSmem<BT>& sm) {
    constexpr int kBW = BT / 32, kBT = BT, kSortTile = BT * kSortItems;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t beg = 0, end = n;
    if constexpr (C > 1) rank_range(n, kSortTile, C, tm.rank, beg, end);
    uint32_t* s_hist = sm.hist;
    uint32_t* s_off = sm.off;
    uint32_t(*s_wcnt)[256] = sm.wcnt;
    for (int pass = 0; pass < 4; ++pass) {
        const uint32_t shift = 8u * pass;
        const uint32_t* kin = s.keys[pass & 1];
        const uint32_t* vin = s.vals[pass & 1];
        uint32_t* kout = s.keys[(pass & 1) ^ 1];
        uint32_t* vout = s.vals[(pass & 1) ^ 1];
        if (threadIdx.x < 256) s_hist[threadIdx.x] = 0;
        __syncthreads();
        for (uint32_t i = beg + threadIdx.x; i < end; i += kBT) atomicAdd(&s_hist[(kin[i] >> shift) & 255u], 1u);
        Team<C>::sync();
        uint32_t hv = 0, below = 0;
        if (threadIdx.x < 256)
            for (uint32_t r = 0; r < uint32_t(C); ++r) {
                const uint32_t v = Team<C>::at(s_hist, r)[threadIdx.x];
                hv += v;
                if (r < tm.rank) below += v;
            }
        uint32_t tot;
        const uint32_t ex = block_scan<BT>(hv, sm.warp, &tot);
        if (threadIdx.x < 256) s_off[threadIdx.x] = ex + below;
        __syncthreads();
        for (uint32_t base = beg; base < end; base += kSortTile) {
            for (int i = threadIdx.x; i < kBW * 256; i += kBT) (&s_wcnt[0][0])[i] = 0;
            __syncthreads();
            uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
#pragma unroll
            for (int j = 0; j < kSortItems; ++j) {
                const uint32_t i = base + warp * (32 * kSortItems) + j * 32 + lane;
                const bool valid = i < end;
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
                if (i < end) {
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
        // the pass's output is complete, and no block reads this block's
        // histogram any more
        Team<C>::sync();
    }
}

// Exclusive scan of c[0..n) into a[0..n), tiles of BT x 8 with a carry; each
// block of the team scans its range, starting from the sum of the lower
// ranks' ranges.
template <int BT, int C>
__device__ void team_scan_array(Team<C> tm, const uint32_t* c, uint32_t* a, uint32_t n, BuildSmem<BT>& sm) {
    constexpr uint32_t kTile = BT * 8;
    uint32_t beg = 0, end = n;
    if constexpr (C > 1) rank_range(n, kTile, C, tm.rank, beg, end);
    uint32_t carry = 0;
    if constexpr (C > 1) {
        uint32_t s = 0, tot;
        for (uint32_t i = beg + threadIdx.x; i < end; i += BT) s += c[i];
        block_scan<BT>(s, sm.warp, &tot);
        if (threadIdx.x == 0) sm.tot = tot;
        Team<C>::sync();
        for (uint32_t r = 0; r < tm.rank; ++r) carry += *Team<C>::at(&sm.tot, r);
    }
    for (uint32_t base = beg; base < end; base += kTile) {
        const uint32_t i0 = base + threadIdx.x * 8;
        uint32_t v[8], sum = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            v[k] = i0 + k < end ? c[i0 + k] : 0u;
            sum += v[k];
        }
        uint32_t tot;
        uint32_t run = carry + block_scan<BT>(sum, sm.warp, &tot);
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (i0 + k < end) a[i0 + k] = run;
            run += v[k];
        }
        carry += tot;
    }
    Team<C>::sync();
}

// One mesh's LBVH build by the team: every per-element step is strided over
// the team's C x BT threads (thread gt), the team meets between steps.
template <int BT, int C>
__device__ __forceinline__ void build_mesh(Team<C> tm, const BuildArgs& A, uint32_t m, BlockScratch& S,
                                       BuildSmem<BT>& sm) {
    constexpr int kBW = BT / 32;
    constexpr uint32_t kGT = uint32_t(C) * BT;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t gt = tm.rank * BT + threadIdx.x;
    const uint32_t n = A.meshes[m].num_triangles;
    // the mesh's arrays, formed where they are used (fewer live registers
    // through the sort)
    auto pos = [&] { return A.pos + size_t(__ldg(&A.meshes[m].vertex_offset)) * A.sf; };
    auto idx = [&] { return A.idx + 3ull * __ldg(&A.meshes[m].triangle_offset); };
    auto toff = [&] { return size_t(__ldg(&A.meshes[m].triangle_offset)); };
    uint32_t* counts = A.counts + 4 * size_t(m);

    // ---- centroids, bounds (per block, then over the team's blocks)
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    {
    const float* vp = pos();
    const uint32_t* ip = idx();
    for (uint32_t t = gt; t < n; t += kGT) {
        rq::F3 p0, p1, p2;
        rq::load_tri(vp, A.sf, ip, t, p0, p1, p2);
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
            sm.red[k][warp] = mn[k];
            sm.red[3 + k][warp] = mx[k];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int k = threadIdx.x;
        float v = sm.red[k][0];
        for (int w = 1; w < kBW; ++w) v = k < 3 ? fminf(v, sm.red[k][w]) : fmaxf(v, sm.red[k][w]);
        sm.bnd[k] = v;
    }
    Team<C>::sync();
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t r = 0; r < uint32_t(C); ++r) {
        const float* b = Team<C>::at(sm.bnd, r);
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], b[k]);
            hi[k] = fmaxf(hi[k], b[3 + k]);
        }
    }
    const float scale = rq::morton_scale(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]);
    for (uint32_t t = gt; t < n; t += kGT) {
        S.keys[0][t] = rq::morton30(S.cent[t], lo[0], lo[1], lo[2], scale);
        S.vals[0][t] = t;
    }
    Team<C>::sync();

    // ---- sort, hierarchy, leaves + refit
    team_sort<BT, C>(tm, S, n, sm);
    for (uint32_t i = gt; i + 1 < n; i += kGT)
        rq::karras_node(S.keys[0], int(n), int(i), S.kl, S.kr, S.klo, S.khi, S.par_in, S.par_lf);
    if (n == 1 && gt == 0) S.par_lf[0] = rq::kNoParent;
    Team<C>::sync();
    for (uint32_t k = gt; k < n; k += kGT) {
        const size_t to = toff();
        rq::leaf_step(k, pos(), A.sf, idx(), A.max_leaf, S.keys[0], S.vals[0], S.klo, S.khi, S.par_in, S.par_lf,
                      S.box_lf, S.c, A.tris + to, A.perm + to, A.skeys + to);
        // a cluster's refit crosses blocks: device-scope arrivals
        rq::refit_walk<C == 1>(k, S.kl, S.kr, S.par_in, S.par_lf, S.box_in, S.box_lf, S.refit_flag, A.err);
    }
    Team<C>::sync();

    // ---- depth-first binary nodes
    team_scan_array<BT, C>(tm, S.c, S.a, n, sm);
    for (uint32_t p = gt; p < n; p += kGT) {
        const uint32_t cp = rq::emit_step(p, n, A.max_leaf, S.kr, S.klo, S.khi, S.par_in, S.par_lf, S.box_in,
                                          S.box_lf, S.c, S.a, A.nodes2 + 2 * toff());
        if (p == n - 1) {
            counts[0] = S.a[p] + cp;
            counts[3] = A.max_leaf;
        }
    }
    Team<C>::sync();

    // ---- 4-wide collapse
    rq::CollapseIO io;
    io.n2 = A.nodes2 + 2 * toff();
    io.q = S.q;
    io.cand = S.cand;
    io.child_q = S.child_q;
    io.sz = S.sz;
    io.par = S.par;
    io.acc = S.acc;
    io.tail = S.tail;
    io.out4 = A.nodes4 + toff();
    io.map4 = A.map4 + 4 * toff();
    uint32_t total = 0, depth = 0;
    auto sync = []() {
        Team<C>::sync();
        return true;
    };
    if (rq::collapse_levels<false, true, 0>(io, gt, kGT, sm.lvl, kMaxLevels, sync, A.err, &total, &depth) &&
        gt == 0) {
        counts[1] = total;
        counts[2] = depth;
    }
    Team<C>::sync();
}

// Meshes order[0, num_big) are built by whole clusters of CL blocks (the
// cluster's first block takes the next one and its scratch slice holds the
// build), the rest by single blocks; every block joins the single-block
// queue once the cluster queue is empty.  CL == 1: no cluster queue.
template <int BT, int CL>
__global__ void __launch_bounds__(BT) k_batch_build(BuildArgs A) {
    __shared__ BuildSmem<BT> sm;
    if constexpr (CL > 1) {
        const uint32_t rank = cg::this_cluster().block_rank();
        BlockScratch S;
        carve_block(reinterpret_cast<uintptr_t>(A.scratch + A.scratch_stride * (blockIdx.x - rank)), A.scratch_n, S);
        for (;;) {
            if (rank == 0 && threadIdx.x == 0) sm.cjob = atomicAdd(A.mesh_ctr, 1u);
            Team<CL>::sync();
            const uint32_t job = *Team<CL>::at(&sm.cjob, 0);
            if (job >= A.num_big) break;
            build_mesh<BT, CL>(Team<CL>{rank}, A, A.order[job], S, sm);
        }
    }
    BlockScratch S;
    carve_block(reinterpret_cast<uintptr_t>(A.scratch + A.scratch_stride * blockIdx.x), A.scratch_n, S);
    for (;;) {
        if (threadIdx.x == 0) sm.job = A.num_big + atomicAdd(A.mesh_ctr + 1, 1u);
        __syncthreads();
        const uint32_t job = sm.job;
        __syncthreads();
        if (job >= A.num_meshes) break;
        build_mesh<BT, 1>(Team<1>{0}, A, A.order[job], S, sm);
    }
    // no block leaves while another may still read its shared memory
    if constexpr (CL > 1) Team<CL>::sync();
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
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_build<BT, 1>, BT, 0) != cudaSuccess) {
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

template <class F>
cudaError_t with_cluster(uint32_t cl, F&& f) {
    if (cl == 2) return f(std::integral_constant<int, 2>{});
    if (cl == 4) return f(std::integral_constant<int, 4>{});
    return f(std::integral_constant<int, 1>{});
}

// Launch configuration of a build shape: `blocks` blocks of BT threads in
// clusters of CL.
struct ClusterLaunch {
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    ClusterLaunch(uint32_t blocks, uint32_t bt, uint32_t cl, cudaStream_t st) {
        cfg.gridDim = dim3(blocks);
        cfg.blockDim = dim3(bt);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = st;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
};

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

int rq_batch_build_clusters(uint32_t threads, uint32_t cluster) {
    if ((threads != 256 && threads != 512 && threads != 1024) || (cluster != 2 && cluster != 4)) return 0;
    int n = 0;
    const cudaError_t e = with_build_shape(threads, [&](auto T) {
        constexpr int BT = decltype(T)::value;
        return with_cluster(cluster, [&](auto L) {
            constexpr int CL = decltype(L)::value;
            ClusterLaunch lc(uint32_t(CL), uint32_t(BT), uint32_t(CL), nullptr);
            return cudaOccupancyMaxActiveClusters(&n, k_batch_build<BT, CL>, &lc.cfg);
        });
    });
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
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
    uint32_t blocks = std::min(b->tune.build_blocks, b->build_slices);
    // clusters: whole clusters within the scratch slices, the meshes of at
    // least cluster_min_tris triangles (the first ones of the size order)
    uint32_t cl = b->tune.build_cluster > 1 ? b->tune.build_cluster : 1u;
    if (cl > 1 && blocks < cl) cl = 1;
    if (cl > 1) blocks -= blocks % cl;
    a.num_big = 0;
    if (cl > 1)
        for (const rq_mesh_desc& d : b->meshes) a.num_big += d.num_triangles >= b->tune.cluster_min_tris ? 1u : 0u;
    cudaError_t e = cudaMemsetAsync(b->d_ctr, 0, 2 * sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = with_build_shape(b->tune.build_threads, [&](auto T) {
            constexpr int BT = decltype(T)::value;
            return with_cluster(cl, [&](auto L) {
                constexpr int CL = decltype(L)::value;
                if constexpr (CL == 1) {
                    k_batch_build<BT, 1><<<blocks, BT, 0, st>>>(a);
                    return cudaGetLastError();
                } else {
                    ClusterLaunch lc(blocks, uint32_t(BT), uint32_t(CL), st);
                    return cudaLaunchKernelEx(&lc.cfg, k_batch_build<BT, CL>, a);
                }
            });
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
