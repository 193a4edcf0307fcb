// k_build.cu — LBVH build of a binary BVH in the layouts of
// common/software_bvh.hpp, one mesh per launch sequence:
//   1. per-triangle centroid ((p0+p1)+p2)/3 (software_bvh.hpp:53) and
//      centroid bounds (ordered-uint atomics);
//   2. 30-bit Morton code in the cube of the largest centroid extent;
//   3. onesweep radix sort of (code, triangle id)              [k_sort.cu]
//   4. Karras 2012 internal nodes, parent links;
//   5. one thread per sorted leaf: leaf-ordered triangle copy, permutation,
//      leaf box, the depth-first emission count of the leaf starting there,
//      then the atomic bottom-up box refit;
//   6. exclusive scan of the emission counts                    [k_sort.cu]
//   7. depth-first pre-order node writes: every emitted node v sits at
//      A[lo(v)] + L(v), where lo(v) is its first primitive, A the scan and
//      L(v) the number of consecutive left-child links above v — the order of
//      SoftwareBVH::recursiveBuild (software_bvh.hpp:90-175): left child at
//      parent + 1, right child after the left subtree;
//   8. the greedy 4-wide collapse                               [k_collapse.cu]
// The per-element steps live in build_core.cuh (shared with k_batch.cu).
// Also the refit of an existing handle (k_parents2, k_refit2, k_refit4).
#include <algorithm>

#include "build_core.cuh"
#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;

__global__ void __launch_bounds__(kT) k_centroids(const float* __restrict__ pos, uint32_t sf,
                                                  const uint32_t* __restrict__ idx, uint32_t n,
                                                  float4* __restrict__ cent, uint32_t* bounds) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = blockIdx.x * kT + threadIdx.x; t < n; t += gridDim.x * kT) {
        rq::F3 p0, p1, p2;
        rq::load_tri(pos, sf, idx, t, p0, p1, p2);
        const float4 c = rq::centroid(p0, p1, p2);
        cent[t] = c;
        mn[0] = fminf(mn[0], c.x);
        mn[1] = fminf(mn[1], c.y);
        mn[2] = fminf(mn[2], c.z);
        mx[0] = fmaxf(mx[0], c.x);
        mx[1] = fmaxf(mx[1], c.y);
        mx[2] = fmaxf(mx[2], c.z);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(&bounds[k], rq::f2o(mn[k]));
            atomicMax(&bounds[3 + k], rq::f2o(mx[k]));
        }
    }
}

__global__ void __launch_bounds__(kT) k_morton(const float4* __restrict__ cent, uint32_t n,
                                               const uint32_t* __restrict__ bounds, uint32_t* __restrict__ keys,
                                               uint32_t* __restrict__ vals) {
    const float lx = rq::o2f(bounds[0]), ly = rq::o2f(bounds[1]), lz = rq::o2f(bounds[2]);
    const float scale = rq::morton_scale(lx, ly, lz, rq::o2f(bounds[3]), rq::o2f(bounds[4]), rq::o2f(bounds[5]));
    for (uint32_t t = blockIdx.x * kT + threadIdx.x; t < n; t += gridDim.x * kT) {
        keys[t] = rq::morton30(cent[t], lx, ly, lz, scale);
        vals[t] = t;
    }
}

__global__ void __launch_bounds__(kT) k_karras(const uint32_t* __restrict__ keys, uint32_t n32,
                                               int32_t* __restrict__ kl, int32_t* __restrict__ kr,
                                               uint32_t* __restrict__ klo, uint32_t* __restrict__ khi,
                                               uint32_t* __restrict__ par_in, uint32_t* __restrict__ par_lf) {
    const int n = int(n32);
    for (int i = blockIdx.x * kT + threadIdx.x; i < n - 1; i += gridDim.x * kT)
        rq::karras_node(keys, n, i, kl, kr, klo, khi, par_in, par_lf);
    if (n == 1 && blockIdx.x == 0 && threadIdx.x == 0) par_lf[0] = rq::kNoParent;
}

// Leaves and refit with the bottom of the tree refitted in shared memory.
// Block b owns the sorted leaves [kLocal*b, kLocal*(b+1)).  A Karras node's
// index is one end of its leaf range, so a node whose range lies inside the
// block's has its index inside it too: such nodes take their arrival count
// and box in shared memory (CTA-scope ordering), and write the box to global
// memory once for the emission.  A walk that reaches a node whose range
// crosses a block boundary stops there and lists its parent link for
// k_refit_top, which carries every such walk on with the device-scope
// acquire-release count of refit_walk: a block is done once its own leaves
// and local nodes are, instead of holding its slot while a walk climbs
// through the tree's top.  Unions are exact, so the boxes equal refit_walk's.
constexpr uint32_t kLocal = 256;  // 17 KB of shared memory per block (measured: faster than 512)

__global__ void __launch_bounds__(kT) k_leaves_local(
    const float* __restrict__ pos, uint32_t sf, const uint32_t* __restrict__ idx, uint32_t n, uint32_t max_leaf,
    const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sids, const int32_t* __restrict__ kl,
    const int32_t* __restrict__ kr, const uint32_t* __restrict__ klo, const uint32_t* __restrict__ khi,
    const uint32_t* __restrict__ par_in, const uint32_t* __restrict__ par_lf, float4* box_in,
    float4* __restrict__ box_lf, uint32_t* refit_flag, uint32_t* __restrict__ c_out, rq_triangle* __restrict__ tris,
    uint32_t* __restrict__ perm, uint32_t* __restrict__ keys_out, uint32_t* __restrict__ top_list,
    uint32_t* top_cnt, uint32_t* err) {
    __shared__ uint32_t s_flag[kLocal];
    __shared__ float4 s_lf[2 * kLocal];  // leaf boxes (lo, hi) of the block's leaves
    __shared__ float4 s_in[2 * kLocal];  // boxes of the block's inner nodes
    __shared__ uint32_t s_top[kLocal];   // the block's handed-over walks (at most one per leaf)
    __shared__ uint32_t s_ntop, s_base;
    const uint32_t L0 = blockIdx.x * kLocal;
    const uint32_t L1 = min(L0 + kLocal, n);
    for (uint32_t i = threadIdx.x; i < kLocal; i += kT) s_flag[i] = 0u;
    if (threadIdx.x == 0) s_ntop = 0u;
    for (uint32_t k = L0 + threadIdx.x; k < L1; k += kT) {
        rq::leaf_step(k, pos, sf, idx, max_leaf, skeys, sids, klo, khi, par_in, par_lf, box_lf, c_out, tris, perm,
                      keys_out);
        s_lf[2 * (k - L0)] = box_lf[2 * size_t(k)];
        s_lf[2 * (k - L0) + 1] = box_lf[2 * size_t(k) + 1];
    }
    __syncthreads();
    for (uint32_t k = L0 + threadIdx.x; k < L1; k += kT) {
        uint32_t par = par_lf[k];
        uint32_t guard = 0;
        while (par != rq::kNoParent) {
            const uint32_t p = par >> 1;
            const int32_t a = kl[p], b = kr[p];
            float4 alo, ahi, blo, bhi;
            if (__ldg(klo + p) >= L0 && __ldg(khi + p) < L1) {
                __threadfence_block();  // release this thread's shared-memory box
                if (atomicAdd(&s_flag[p - L0], 1u) == 0u) break;
                __threadfence_block();  // acquire the sibling's
                const float4* pa = a < 0 ? s_lf + 2 * ((uint32_t(a) & 0x7fffffffu) - L0) : s_in + 2 * (a - L0);
                const float4* pb = b < 0 ? s_lf + 2 * ((uint32_t(b) & 0x7fffffffu) - L0) : s_in + 2 * (b - L0);
                alo = pa[0];
                ahi = pa[1];
                blo = pb[0];
                bhi = pb[1];
                const float4 lo = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f);
                const float4 hi = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f);
                s_in[2 * (p - L0)] = lo;
                s_in[2 * (p - L0) + 1] = hi;
                __stcg(box_in + 2 * size_t(p), lo);
                __stcg(box_in + 2 * size_t(p) + 1, hi);
            } else {
                // from here up every range crosses a block boundary: k_refit_top
                s_top[atomicAdd(&s_ntop, 1u)] = par;
                break;
            }
            par = par_in[p];
            if (++guard > 128u) {
                rq::set_err(err, RQ_DERR_REFIT);
                break;
            }
        }
    }
    // the block's hand-offs, with one device atomic
    __syncthreads();
    const uint32_t nt = s_ntop;
    if (threadIdx.x == 0 && nt) s_base = atomicAdd(top_cnt, nt);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < nt; i += kT) top_list[s_base + i] = s_top[i];
}

// The walks k_leaves_local handed over: each starts at the parent link of a
// node whose parent's range crosses a block boundary (that node's box is in
// box_in or box_lf); at each node the second child to arrive forms the union
// and carries on upward, as refit_walk.
__global__ void __launch_bounds__(kT) k_refit_top(const int32_t* __restrict__ kl, const int32_t* __restrict__ kr,
                                                  const uint32_t* __restrict__ par_in, float4* box_in,
                                                  const float4* box_lf, uint32_t* refit_flag,
                                                  const uint32_t* __restrict__ top_list, const uint32_t* top_cnt,
                                                  uint32_t* err) {
    const uint32_t m = *top_cnt;
    for (uint32_t j = blockIdx.x * kT + threadIdx.x; j < m; j += gridDim.x * kT) {
        uint32_t par = top_list[j];
        uint32_t guard = 0;
        while (par != rq::kNoParent) {
            const uint32_t p = par >> 1;
            if (rq::atom_add_acq_rel(&refit_flag[p], 1u) == 0u) break;
            const int32_t a = kl[p], b = kr[p];
            const float4* ba = a < 0 ? box_lf + 2 * size_t(uint32_t(a) & 0x7fffffffu) : box_in + 2 * size_t(a);
            const float4* bb = b < 0 ? box_lf + 2 * size_t(uint32_t(b) & 0x7fffffffu) : box_in + 2 * size_t(b);
            const float4 alo = rq::ld_cg4(ba), ahi = rq::ld_cg4(ba + 1);
            const float4 blo = rq::ld_cg4(bb), bhi = rq::ld_cg4(bb + 1);
            __stcg(box_in + 2 * size_t(p),
                   make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f));
            __stcg(box_in + 2 * size_t(p) + 1,
                   make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f));
            par = par_in[p];
            if (++guard > 128u) {
                rq::set_err(err, RQ_DERR_REFIT);
                break;
            }
        }
    }
}

__global__ void __launch_bounds__(kT) k_emit2(uint32_t n, uint32_t max_leaf, const int32_t* __restrict__ kr,
                                              const uint32_t* __restrict__ klo, const uint32_t* __restrict__ khi,
                                              const uint32_t* __restrict__ par_in,
                                              const uint32_t* __restrict__ par_lf, const float4* __restrict__ box_in,
                                              const float4* __restrict__ box_lf, const uint32_t* __restrict__ c,
                                              const uint32_t* __restrict__ A, rq_bvh2_node* __restrict__ out,
                                              uint32_t* __restrict__ counts) {
    for (uint32_t p = blockIdx.x * kT + threadIdx.x; p < n; p += gridDim.x * kT) {
        const uint32_t cp = rq::emit_step(p, n, max_leaf, kr, klo, khi, par_in, par_lf, box_in, box_lf, c, A, out);
        if (p == n - 1) {
            counts[0] = A[p] + cp;  // binary node count
            counts[3] = max_leaf;
        }
    }
}

// ------------------------------------------------- SAH-rebuilt subtrees
// RQ_BUILD_SAH: the Karras hierarchy above every node of at most K
// primitives stays; each such subtree (a contiguous range of the sorted
// order) is rebuilt top down by binned SAH inside one block: B bins per axis
// over the node's centroid bounds (B = 16 above kSahSmallNode primitives, 8 at
// or below), bin = min(B - 1, int((c - cmin) * (B / extent))), cost
// float(nL) * SA(left) + float(nR) * SA(right), the smallest
// cost first by axis then bin, a stable partition of the node's range, leaves
// of at most max_leaf primitives, the middle of the range where no axis has
// a centroid extent or the subtree is kSahDepthCap levels deep.  Every node
// still covers a contiguous range of leaf positions, so the pre-order
// position of every node is A[lo(v)] + L(v) as in the plain LBVH: the subtree
// blocks write one record per node (box, first position, L, and the right
// child's first position or the leaf count) and the emission counts of their
// leaves; after the scan, k_sah_emit writes the records and the top nodes.
constexpr uint32_t kSahMax = 1024;  // largest subtree a block rebuilds in shared memory
constexpr uint32_t kSahNone = 0xffffffffu;  // no Karras node above (no top refit from here)
constexpr int kSahT = 256;
constexpr int kSahWarps = kSahT / 32;
// Nodes of more than kSahSmallNode primitives are binned 16 ways per axis,
// smaller ones 8 ways (as good for the small nodes, at half the pricing).
constexpr uint32_t kSahSmallNode = 32;
template <int NB>
struct SahBinsOf {
    static constexpr uint32_t slots = 3u * NB;       // (axis, bin) pairs of one node
    static constexpr uint32_t words = 7u * slots;    // count, min xyz, max xyz: field-major
    static constexpr int axes_per_pass = 32 / NB;    // axes one warp prices at a time
    static_assert(words % 4u == 0u && slots % 4u == 0u, "bins are cleared with 16-byte stores");
};
constexpr uint32_t kSahDepthCap = 24;
// depths at which a node of more than kSahMax triangles can lie (the queue's capacity)
constexpr uint32_t kSahMidDepths = kSahDepthCap + 8u;
static_assert(RQ_SAH_SUBTREE_MAX <= 64u * kSahMax, "kSahMidDepths allows 6 halvings after the SAH levels");
constexpr uint32_t kNoRecord = 0xffffffffu;

// Per sorted position: the triangle's box with its x and y centroid in w, its
// z centroid, and the identity order (the order of every SAH root at depth 0).
__global__ void __launch_bounds__(kT) k_sah_pbox(const float* __restrict__ pos, uint32_t sf,
                                                 const uint32_t* __restrict__ idx, uint32_t n,
                                                 const uint32_t* __restrict__ sids, const float4* __restrict__ cent,
                                                 float4* __restrict__ plo, float4* __restrict__ phi,
                                                 float* __restrict__ pcz, uint32_t* __restrict__ ord0) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const uint32_t gid = sids[i];
        rq::F3 p0, p1, p2;
        rq::load_tri(pos, sf, idx, gid, p0, p1, p2);
        const float4 c = cent[gid];
        plo[i] = make_float4(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)),
                             fminf(p0.z, fminf(p1.z, p2.z)), c.x);
        phi[i] = make_float4(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)),
                             fmaxf(p0.z, fmaxf(p1.z, p2.z)), c.y);
        pcz[i] = c.z;
        ord0[i] = i;
    }
}

// Where a finished SAH root's subtree goes next: a block subtree (at most
// kSahMax triangles: recorded at its first sorted position — last position,
// left-child links above it, depth, Karras node above or kSahNone — and
// appended to the block list) or the node queue of k_sah_mid.
struct SahOut {
    uint32_t* list;
    uint32_t* count;
    uint32_t* shi;
    uint32_t* sL;
    uint32_t* sdepth;
    uint32_t* snode;
    uint4* mq;
    uint32_t* mready;
    uint32_t mcap;
    uint32_t* ctl;
    uint32_t* err;
};

// bnd (queue entries only, may be null): the node's bounds, 12 floats: box
// min, box max, centroid min, centroid max.  A queue entry is 4 uint4: s, e,
// depth | L << 8, Karras node; then the bounds; its written flag is 2 with the
// bounds, 1 without.
__device__ __forceinline__ void sah_route(const SahOut& O, uint32_t s, uint32_t e, uint32_t depth, uint32_t L,
                                          uint32_t node, const float* bnd = nullptr) {
    if (e - s <= kSahMax) {
        O.shi[s] = e - 1u;
        O.sL[s] = L;
        O.sdepth[s] = depth;
        O.snode[s] = node;
        O.list[atomicAdd(O.count, 1u)] = s;
        return;
    }
    const uint32_t k = atomicAdd(O.ctl + 1, 1u);
    if (k >= O.mcap) {  // cannot happen (the queue holds every node of more than kSahMax)
        rq::set_err(O.err, RQ_DERR_QUEUE);
        return;
    }
    uint4* q = O.mq + 4 * size_t(k);
    __stcg(q, make_uint4(s, e, depth | (L << 8), node));
    if (bnd) {
#pragma unroll
        for (int j = 0; j < 3; ++j)
            __stcg(q + 1 + j, make_uint4(__float_as_uint(bnd[4 * j]), __float_as_uint(bnd[4 * j + 1]),
                                         __float_as_uint(bnd[4 * j + 2]), __float_as_uint(bnd[4 * j + 3])));
    }
    __threadfence();
    rq::st_release(O.mready + k, bnd ? 2u : 1u);
}

// SAH roots: every child of at most K primitives of a Karras node of more (or
// the root itself when n <= K), in any order (a subtree's output depends on
// its own primitives only), routed with the left-child links above it and its
// Karras node.
__global__ void __launch_bounds__(kT) k_sah_roots(uint32_t n, uint32_t K, const int32_t* __restrict__ kl,
                                                  const int32_t* __restrict__ kr, const uint32_t* __restrict__ klo,
                                                  const uint32_t* __restrict__ khi,
                                                  const uint32_t* __restrict__ par_in, SahOut O) {
    if (n <= K) {
        if (blockIdx.x == 0 && threadIdx.x == 0) sah_route(O, 0u, n, 0u, 0u, n == 1u ? 0x80000000u : 0u);
        return;
    }
    for (uint32_t p = blockIdx.x * kT + threadIdx.x; p + 1u < n; p += gridDim.x * kT) {
        if (rq::count_in(klo, khi, p) <= K) continue;
        uint32_t L = 0, par = par_in[p];
        while (par != rq::kNoParent && (par & 1u) == 0u) {
            ++L;
            par = par_in[par >> 1];
        }
        const int32_t ch[2] = {kl[p], kr[p]};
#pragma unroll
        for (int side = 0; side < 2; ++side) {
            const bool leaf = ch[side] < 0;
            const uint32_t ci = uint32_t(ch[side]) & 0x7fffffffu;
            const uint32_t lo = leaf ? ci : klo[ci], hi = leaf ? ci : khi[ci];
            if (hi - lo + 1u > K) continue;
            sah_route(O, lo, hi + 1u, 0u, side == 0 ? L + 1u : 0u, leaf ? (0x80000000u | ci) : ci);
        }
    }
}

// A finished SAH root's box where its Karras parent's union reads it, then the
// walk up the Karras nodes above it (the second arrival at a node computes its
// box, as refit_walk).  One thread.
__device__ void sah_refit_up(uint32_t rn, float4 rlo, float4 rhi, const int32_t* __restrict__ kl,
                             const int32_t* __restrict__ kr, const uint32_t* __restrict__ par_in,
                             const uint32_t* __restrict__ par_lf, float4* box_in, float4* box_lf,
                             uint32_t* refit_flag, uint32_t* err) {
    const bool rleaf = (rn >> 31) != 0u;
    const uint32_t ri = rn & 0x7fffffffu;
    float4* dst = rleaf ? box_lf + 2 * size_t(ri) : box_in + 2 * size_t(ri);
    __stcg(dst, rlo);
    __stcg(dst + 1, rhi);
    uint32_t par = rleaf ? par_lf[ri] : par_in[ri];
    for (uint32_t guard = 0; par != rq::kNoParent; ++guard) {
        const uint32_t p = par >> 1;
        if (rq::atom_add_acq_rel(&refit_flag[p], 1u) == 0u) break;
        const int32_t a = kl[p], b = kr[p];
        const float4* ba = a < 0 ? box_lf + 2 * size_t(uint32_t(a) & 0x7fffffffu) : box_in + 2 * size_t(a);
        const float4* bb = b < 0 ? box_lf + 2 * size_t(uint32_t(b) & 0x7fffffffu) : box_in + 2 * size_t(b);
        const float4 alo = rq::ld_cg4(ba), ahi = rq::ld_cg4(ba + 1), blo = rq::ld_cg4(bb), bhi = rq::ld_cg4(bb + 1);
        __stcg(box_in + 2 * size_t(p), make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f));
        __stcg(box_in + 2 * size_t(p) + 1,
               make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f));
        par = par_in[p];
        if (guard > 128u) {
            rq::set_err(err, RQ_DERR_REFIT);
            break;
        }
    }
}

struct SahArgs {
    uint32_t n, max_leaf;
    const float4* plo;  // per sorted position: box min, centroid x
    const float4* phi;  // box max, centroid y
    const float* pcz;   // centroid z
    const uint32_t* ord[2];  // the order of the sorted positions at even / odd depths
    const uint32_t* sdepth;
    const float* pos;
    uint32_t sf;
    const uint32_t* idx;
    const uint32_t* skeys;
    const uint32_t* sids;
    const int32_t* kl;
    const int32_t* kr;
    const uint32_t* par_in;
    const uint32_t* par_lf;
    float4* box_in;
    float4* box_lf;
    uint32_t* refit_flag;
    const uint32_t* shi;
    const uint32_t* sL;
    const uint32_t* snode;
    const uint32_t* list;
    const uint32_t* count;
    uint32_t* next;
    float4* rec;
    uint32_t* rec_l;
    uint32_t* c;
    rq_triangle* tris;
    uint32_t* perm;
    uint32_t* keys_out;
    uint32_t* err;
};

// Shared memory of one subtree block (kSahMax primitives): boxes with the x
// and y centroid in w, z centroids, triangle ids, the leaf order at even and
// odd depths and the final one (local indices), the node lists of two levels,
// and one set of bins per warp (7 fields x 3 axes x 16 bins: count, min xyz,
// max xyz as ordered integers, field-major).
struct SahShared {
    float4 lo[kSahMax];
    float4 hi[kSahMax];
    float cz[kSahMax];
    uint32_t id[kSahMax];
    uint16_t ord[2][kSahMax];
    uint16_t fin[kSahMax];  // the final leaf order: each leaf writes its range
    uint2 list[2][kSahMax];
    alignas(16) uint32_t bins[kSahWarps][SahBinsOf<16>::words];
    uint32_t cnt[2];
    uint32_t slots;
    uint32_t job;
    float4 root_lo, root_hi;
};

// int((c - cmin) * scale) for a centroid c of the node: the product lies in
// [0, ~bins] (scale = bins / the node's extent), and for x in [0, 2^23) the
// sum 2^23 + x rounded toward zero is 2^23 + floor(x), so its low mantissa
// bits are the truncation (an FADD instead of a float-to-int conversion, which
// issues at a quarter of the rate).
__device__ __forceinline__ uint32_t sah_floor(float c, float cmin, float scale) {
    return __float_as_uint(__fadd_rz((c - cmin) * scale, 8388608.0f)) & 0x7fffffu;
}

// The bin: the truncation clamped to the last of NB bins.
template <int NB>
__device__ __forceinline__ uint32_t sah_bin(float c, float cmin, float scale) {
    const uint32_t b = sah_floor(c, cmin, scale);
    return b < uint32_t(NB - 1) ? b : uint32_t(NB - 1);
}

__device__ __forceinline__ float sah_area(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    const float dx = mxx - mnx, dy = mxy - mny, dz = mxz - mnz;
    return 2.0f * ((dx * dy + dy * dz) + dz * dx);
}

__device__ __forceinline__ float sah_pick(const float (&v)[3], int a) {
    return a == 0 ? v[0] : (a == 1 ? v[1] : v[2]);
}

__device__ __forceinline__ float sah_centroid(const SahShared& S, uint32_t p, int a) {
    return a == 0 ? S.lo[p].w : (a == 1 ? S.hi[p].w : S.cz[p]);
}

// Node list entry: x = s | e << 11 | depth << 22, y = slot | boxed << 11 |
// L << 12 (slot: the node's record slot, below 2 x kSahMax; boxed: the
// parent wrote the node's box into its record; L: the consecutive left-child
// links above it).
__device__ __forceinline__ uint2 sah_entry(uint32_t s, uint32_t e, uint32_t depth, uint32_t slot, uint32_t L,
                                           bool boxed = false) {
    return make_uint2(s | (e << 11) | (depth << 22), slot | (boxed ? 0x800u : 0u) | (L << 12));
}

// Record r's box (min xyz, max xyz) without its w words, and its w words
// (first position; right child's first position or bit 31 | leaf count)
// without the box: a parent that knows a child's box writes the one, the
// child the other.
__device__ __forceinline__ void sah_rec_box(float4* rec, size_t r, const float (&b)[6]) {
    float* f = reinterpret_cast<float*>(rec + 2 * r);
    f[0] = b[0];
    f[1] = b[1];
    f[2] = b[2];
    f[4] = b[3];
    f[5] = b[4];
    f[6] = b[5];
}
__device__ __forceinline__ void sah_rec_aux(float4* rec, size_t r, uint32_t first, uint32_t aux) {
    float* f = reinterpret_cast<float*>(rec + 2 * r);
    f[3] = __uint_as_float(first);
    f[7] = __uint_as_float(aux);
}

// The bins of one node (7 fields x 3 axes x NB bins, field-major: count,
// min xyz, max xyz as ordered integers), cleared by one warp with 16-byte
// stores (a field is a whole number of them).
template <int NB>
__device__ __forceinline__ void sah_bins_clear(uint32_t* bins, uint32_t lane) {
    using B = SahBinsOf<NB>;
    uint4* b4 = reinterpret_cast<uint4*>(bins);
    for (uint32_t w = lane; w < B::words / 4u; w += 32) {
        const uint32_t f = w / (B::slots / 4u);
        const uint32_t v = f == 0 ? 0u : (f <= 3 ? rq::f2o(INFINITY) : rq::f2o(-INFINITY));
        b4[w] = make_uint4(v, v, v, v);
    }
}

// NB / extent per axis, 0 where the centroids have no extent or the extent is
// too small to scale (no split on that axis).  Called by a whole warp with
// the same bounds in every lane: lane a < 3 divides for axis a, one division
// per lane instead of three.
template <int NB>
__device__ __forceinline__ void sah_scales(const float (&cmn)[3], const float (&cmx)[3], float (&scale)[3],
                                           uint32_t lane) {
    const int a = lane < 3u ? int(lane) : 0;
    const float ext = sah_pick(cmx, a) - sah_pick(cmn, a);
    float sc = ext > 0.0f ? float(NB) / ext : 0.0f;
    if (!(sc < INFINITY)) sc = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) scale[k] = __shfl_sync(0xffffffffu, sc, k);
}

// Bins the primitives at ord[s, e) into `bins` (one warp).  Each lane bins a
// run of C consecutive primitives: consecutive primitives are close in space
// and mostly share a bin, so lanes on far-apart runs update different bins
// (with the lanes on consecutive primitives, the warp's atomics serialise on
// one address).  C is odd, so the 16-byte box loads of 8 lanes at stride C
// fall in distinct banks.
template <int NB>
__device__ __forceinline__ void sah_bin_range(const SahShared& S, uint32_t* bins, const uint16_t* ord, uint32_t s,
                                              uint32_t e, uint32_t lane, const float (&cmn)[3],
                                              const float (&scale)[3]) {
    const uint32_t run = ((e - s + 31u) >> 5) | 1u;
    for (uint32_t j = 0; j < run; ++j) {
        const uint32_t i = s + lane * run + j;
        if (i >= e) break;
        const uint32_t p = ord[i];
        const float4 a4 = S.lo[p], b4 = S.hi[p];
        const float c[3] = {a4.w, b4.w, S.cz[p]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (!(scale[a] > 0.0f)) continue;
            constexpr uint32_t F = SahBinsOf<NB>::slots;
            uint32_t* bn = bins + a * NB + sah_bin<NB>(c[a], cmn[a], scale[a]);
            atomicAdd(bn, 1u);
            atomicMin(bn + 1 * F, rq::f2o(a4.x));
            atomicMin(bn + 2 * F, rq::f2o(a4.y));
            atomicMin(bn + 3 * F, rq::f2o(a4.z));
            atomicMax(bn + 4 * F, rq::f2o(b4.x));
            atomicMax(bn + 5 * F, rq::f2o(b4.y));
            atomicMax(bn + 6 * F, rq::f2o(b4.z));
        }
    }
}

// The split of the filled bins (one warp, every lane gets the result):
// 3 x (NB - 1) candidates (axis, split after bin k).  32 / NB axes per pass,
// one per lane segment, lane b of a segment holding bin b: inclusive prefix
// and suffix unions over the bins (min / max are exact, so the unions equal
// any other order's), then lane k < NB - 1 prices the split after bin k.  The
// winner is the smallest finite cost, the lowest candidate among equal costs.
// axis < 0: no split.
template <int NB>
__device__ __forceinline__ void sah_choose(const uint32_t* bins, const float (&scale)[3], uint32_t lane, int& axis,
                                           int& split, uint32_t& nl_out, float (&lbox)[6], float (&rbox)[6]) {
    constexpr uint32_t F = SahBinsOf<NB>::slots;
    float bc = INFINITY;
    uint32_t bi = 0xffffffffu, bnl = 0;
    float blb[6], brb[6];  // this lane's best candidate's left and right boxes
#pragma unroll
    for (int q = 0; q < 6; ++q) blb[q] = brb[q] = 0.0f;
    for (int pass = 0; pass * SahBinsOf<NB>::axes_per_pass < 3; ++pass) {
        const int a = pass * SahBinsOf<NB>::axes_per_pass + int(lane / NB);
        const uint32_t b = lane % NB;
        const bool live = a < 3 && sah_pick(scale, a) > 0.0f;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t cnt = 0;
        if (live) {
            const uint32_t* bn = bins + a * NB + b;
            cnt = bn[0];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                lo[q] = rq::o2f(bn[(1 + q) * F]);
                hi[q] = rq::o2f(bn[(4 + q) * F]);
            }
        }
        float plo[3] = {lo[0], lo[1], lo[2]}, phi[3] = {hi[0], hi[1], hi[2]};
        float slo[3] = {lo[0], lo[1], lo[2]}, shi[3] = {hi[0], hi[1], hi[2]};
        uint32_t pc = cnt, sc = cnt;
#pragma unroll
        for (int o = 1; o < NB; o <<= 1) {
            const uint32_t upc = __shfl_up_sync(0xffffffffu, pc, o, NB);
            const uint32_t dnc = __shfl_down_sync(0xffffffffu, sc, o, NB);
            float u[6], d[6];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                u[q] = __shfl_up_sync(0xffffffffu, plo[q], o, NB);
                u[3 + q] = __shfl_up_sync(0xffffffffu, phi[q], o, NB);
                d[q] = __shfl_down_sync(0xffffffffu, slo[q], o, NB);
                d[3 + q] = __shfl_down_sync(0xffffffffu, shi[q], o, NB);
            }
            if (b >= uint32_t(o)) {
                pc += upc;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    plo[q] = fminf(plo[q], u[q]);
                    phi[q] = fmaxf(phi[q], u[3 + q]);
                }
            }
            if (b + uint32_t(o) < uint32_t(NB)) {
                sc += dnc;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    slo[q] = fminf(slo[q], d[q]);
                    shi[q] = fmaxf(shi[q], d[3 + q]);
                }
            }
        }
        // the right side of split b is the suffix from bin b + 1
        const uint32_t nr = __shfl_down_sync(0xffffffffu, sc, 1, NB);
        float r[6];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            r[q] = __shfl_down_sync(0xffffffffu, slo[q], 1, NB);
            r[3 + q] = __shfl_down_sync(0xffffffffu, shi[q], 1, NB);
        }
        if (live && b < uint32_t(NB - 1)) {
            const float cost = float(pc) * sah_area(plo[0], plo[1], plo[2], phi[0], phi[1], phi[2]) +
                               float(nr) * sah_area(r[0], r[1], r[2], r[3], r[4], r[5]);
            const uint32_t cand = uint32_t(a) * (NB - 1) + b;
            if (cost < bc) {
                bc = cost;
                bi = cand;
                bnl = pc;
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    blb[q] = plo[q];
                    blb[3 + q] = phi[q];
                    brb[q] = r[q];
                    brb[3 + q] = r[3 + q];
                }
            }
        }
    }
    // The smallest (cost, candidate): costs are +0, positive or +inf, so
    // their bits order as their values.
    const uint32_t cbits = __float_as_uint(bc);
    const uint32_t cmin = __reduce_min_sync(0xffffffffu, cbits);
    const uint32_t mine = cbits == cmin ? bi : 0xffffffffu;
    const uint32_t win = __reduce_min_sync(0xffffffffu, mine);
    const uint32_t holder = __ballot_sync(0xffffffffu, win != 0xffffffffu && mine == win);
    const uint32_t hl = holder ? uint32_t(__ffs(holder) - 1) : 0u;
    bnl = __shfl_sync(0xffffffffu, bnl, hl);
    // the winner's prefix and suffix unions: exactly the children's boxes
    // (min and max are exact in any order)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        lbox[q] = __shfl_sync(0xffffffffu, blb[q], hl);
        rbox[q] = __shfl_sync(0xffffffffu, brb[q], hl);
    }
    axis = -1;
    split = -1;
    nl_out = 0;
    if (win != 0xffffffffu) {
        axis = int(win / (NB - 1));
        split = int(win % (NB - 1));
        nl_out = bnl;
    }
}

// The binned split of a node (one warp): clear the warp's bins, bin the
// node's primitives, price the candidates; the chosen axis's scale for the
// partition.
template <int NB>
__device__ __forceinline__ void sah_split(const SahShared& S, uint32_t* bins, const uint16_t* ord, uint32_t s,
                                          uint32_t e, uint32_t lane, const float (&cmn)[3], const float (&cmx)[3],
                                          int& axis, int& split, uint32_t& nl, float& axis_scale,
                                          float (&lbox)[6], float (&rbox)[6]) {
    float scale[3];
    sah_bins_clear<NB>(bins, lane);
    sah_scales<NB>(cmn, cmx, scale, lane);
    __syncwarp();
    sah_bin_range<NB>(S, bins, ord, s, e, lane, cmn, scale);
    __syncwarp();
    sah_choose<NB>(bins, scale, lane, axis, split, nl, lbox, rbox);
    __syncwarp();  // the bins are read before the next node reuses them
    axis_scale = axis < 0 ? 0.0f : sah_pick(scale, axis);
}

// Centroid bounds over a warp in every lane: warp min / max reductions of the
// values as order-preserving integers (exact, as any min / max).  Lanes
// without a primitive contribute the identities (+inf for the minimum,
// -inf for the maximum).
__device__ __forceinline__ void sah_warp_bounds2(const float (&lmn)[3], const float (&lmx)[3], float (&cmn)[3],
                                                 float (&cmx)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        cmn[k] = rq::o2f(__reduce_min_sync(0xffffffffu, rq::f2o(lmn[k])));
        cmx[k] = rq::o2f(__reduce_max_sync(0xffffffffu, rq::f2o(lmx[k])));
    }
}
__device__ __forceinline__ void sah_warp_bounds(const float (&c)[3], bool in, float (&cmn)[3], float (&cmx)[3]) {
    const float lmn[3] = {in ? c[0] : INFINITY, in ? c[1] : INFINITY, in ? c[2] : INFINITY};
    const float lmx[3] = {in ? c[0] : -INFINITY, in ? c[1] : -INFINITY, in ? c[2] : -INFINITY};
    sah_warp_bounds2(lmn, lmx, cmn, cmx);
}

// A node of at most 32 primitives (every leaf, and most inner nodes), by one
// warp with lane i holding primitive s + i: the same bounds, 8-way bins,
// pricing and stable partition as sah_node's loops, without the loops.
// boxed: the parent wrote this node's box into its record (no box
// reduction here).  After a binned split the children's boxes are the
// winning candidate's unions: they go into the children's records, and a
// child of at most max_leaf primitives is written as a leaf here (record,
// final order, emission count) instead of being listed.  Returns the
// children to list (bit 0 left, bit 1 right).
__device__ __forceinline__ uint32_t sah_node_small(SahShared& S, const SahArgs& A, uint32_t lo, uint32_t s, uint32_t n,
                                                   uint32_t depth, uint32_t slot, uint32_t L, bool boxed,
                                                   uint32_t lane, uint32_t warp, uint2& left_child,
                                                   uint2& right_child) {
    static_assert(kSahSmallNode == 32u, "one primitive per lane");
    const uint16_t* ord = S.ord[depth & 1u];
    uint16_t* nxt = S.ord[(depth + 1u) & 1u];
    const bool in = lane < n;
    const uint32_t p = ord[s + (in ? lane : 0u)];
    const float4 a = S.lo[p], b = S.hi[p];
    float mn[3] = {in ? a.x : INFINITY, in ? a.y : INFINITY, in ? a.z : INFINITY};
    float mx[3] = {in ? b.x : -INFINITY, in ? b.y : -INFINITY, in ? b.z : -INFINITY};
    const size_t r = 2ull * lo + slot;  // record index
    if (!boxed) {
        // butterfly over lanes 0..n-1 (the others hold the identities): the bounds end in lane 0
        for (uint32_t o = 1; o < n; o <<= 1)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
            }
        if (slot == 0 && lane == 0) {  // the subtree root's box, for the top refit
            S.root_lo = make_float4(mn[0], mn[1], mn[2], 0.0f);
            S.root_hi = make_float4(mx[0], mx[1], mx[2], 0.0f);
        }
    }
    if (n <= A.max_leaf) {
        if (lane == 0) {
            if (boxed) {
                sah_rec_aux(A.rec, r, lo + s, 0x80000000u | n);
            } else {
                A.rec[2 * r] = make_float4(mn[0], mn[1], mn[2], __uint_as_float(lo + s));
                A.rec[2 * r + 1] = make_float4(mx[0], mx[1], mx[2], __uint_as_float(0x80000000u | n));
            }
            A.rec_l[r] = L;
        }
        // the triangles are written once the subtree is done (sah_leaves)
        if (in) {
            S.fin[s + lane] = uint16_t(p);
            A.c[lo + s + lane] = lane == 0 ? 1u + L : 0u;
        }
        return 0u;
    }
    const float c[3] = {a.w, b.w, S.cz[p]};
    float cmn[3], cmx[3];
    sah_warp_bounds(c, in, cmn, cmx);
    int best_axis = -1, best_split = -1;
    uint32_t best_nl = 0;
    float scale[3] = {0.0f, 0.0f, 0.0f};
    float lbox[6], rbox[6];
    if (depth < kSahDepthCap) {
        uint32_t* bins = S.bins[warp];
        sah_bins_clear<8>(bins, lane);
        sah_scales<8>(cmn, cmx, scale, lane);
        __syncwarp();
        if (in) {
            constexpr uint32_t F = SahBinsOf<8>::slots;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (!(scale[k] > 0.0f)) continue;
                uint32_t* bn = bins + k * 8 + sah_bin<8>(c[k], cmn[k], scale[k]);
                atomicAdd(bn, 1u);
                atomicMin(bn + 1 * F, rq::f2o(a.x));
                atomicMin(bn + 2 * F, rq::f2o(a.y));
                atomicMin(bn + 3 * F, rq::f2o(a.z));
                atomicMax(bn + 4 * F, rq::f2o(b.x));
                atomicMax(bn + 5 * F, rq::f2o(b.y));
                atomicMax(bn + 6 * F, rq::f2o(b.z));
            }
        }
        __syncwarp();
        sah_choose<8>(bins, scale, lane, best_axis, best_split, best_nl, lbox, rbox);
        __syncwarp();  // the bins are read before the next node reuses them
    }
    const bool known = best_axis >= 0;  // the children's boxes are lbox, rbox
    uint32_t mid;
    bool leaf_l = false, leaf_r = false;
    if (!known) {
        mid = s + n / 2u;
        if (in) nxt[s + lane] = uint16_t(p);
    } else {
        mid = s + best_nl;
        leaf_l = mid - s <= A.max_leaf;
        leaf_r = s + n - mid <= A.max_leaf;
        // the clamp to the last bin cannot move a centroid across a split
        const bool left = in && sah_floor(sah_pick(c, best_axis), sah_pick(cmn, best_axis),
                                          sah_pick(scale, best_axis)) <= uint32_t(best_split);
        const uint32_t lt = (1u << lane) - 1u;
        const uint32_t ml = __ballot_sync(0xffffffffu, left), mr = __ballot_sync(0xffffffffu, in && !left);
        if (left) {
            const uint32_t q = s + __popc(ml & lt);
            nxt[q] = uint16_t(p);
            if (leaf_l) {  // the left child's leaf: final order and emission count (L + 1 left links)
                S.fin[q] = uint16_t(p);
                A.c[lo + q] = q == s ? 2u + L : 0u;
            }
        } else if (in) {
            const uint32_t q = mid + __popc(mr & lt);
            nxt[q] = uint16_t(p);
            if (leaf_r) {  // the right child's leaf (no left link above it)
                S.fin[q] = uint16_t(p);
                A.c[lo + q] = q == mid ? 1u : 0u;
            }
        }
    }
    uint32_t cs = 0;
    if (lane == 0) {
        if (boxed) {
            sah_rec_aux(A.rec, r, lo + s, lo + mid);
        } else {
            A.rec[2 * r] = make_float4(mn[0], mn[1], mn[2], __uint_as_float(lo + s));
            A.rec[2 * r + 1] = make_float4(mx[0], mx[1], mx[2], __uint_as_float(lo + mid));
        }
        A.rec_l[r] = L;
        cs = atomicAdd(&S.slots, 2u);
        if (known) {
            const size_t rl = 2ull * lo + cs, rr = rl + 1;
            if (leaf_l) {
                A.rec[2 * rl] = make_float4(lbox[0], lbox[1], lbox[2], __uint_as_float(lo + s));
                A.rec[2 * rl + 1] = make_float4(lbox[3], lbox[4], lbox[5], __uint_as_float(0x80000000u | (mid - s)));
                A.rec_l[rl] = L + 1u;
            } else {
                sah_rec_box(A.rec, rl, lbox);
            }
            if (leaf_r) {
                A.rec[2 * rr] = make_float4(rbox[0], rbox[1], rbox[2], __uint_as_float(lo + mid));
                A.rec[2 * rr + 1] =
                    make_float4(rbox[3], rbox[4], rbox[5], __uint_as_float(0x80000000u | (s + n - mid)));
                A.rec_l[rr] = 0u;
            } else {
                sah_rec_box(A.rec, rr, rbox);
            }
        }
    }
    cs = __shfl_sync(0xffffffffu, cs, 0);
    left_child = sah_entry(s, mid, depth + 1u, cs, L + 1u, known);
    right_child = sah_entry(mid, s + n, depth + 1u, cs + 1u, 0u, known);
    return (leaf_l ? 0u : 1u) | (leaf_r ? 0u : 2u);
}

// One node of a subtree, by one warp: box and centroid bounds, then a leaf
// (its record, emission counts, triangles; returns false) or the binned
// split: the stable partition of its range into the order of the next depth,
// its record, and its two children in every lane (returns true).  A node at
// depth d reads ord[d & 1] and writes ord[(d + 1) & 1] over its own range:
// ranges of nodes that are not ancestors of one another are disjoint, and a
// node's range is complete before its children start.  Returns the children
// to list (bit 0 left, bit 1 right); a node with a binned split writes its
// children's boxes into their records (their entries are boxed).
__device__ uint32_t sah_node(SahShared& S, const SahArgs& A, uint32_t lo, uint2 ent, uint32_t lane, uint32_t warp,
                             uint2& left_child, uint2& right_child) {
    const uint32_t s = ent.x & 0x7ffu, e = (ent.x >> 11) & 0x7ffu, depth = ent.x >> 22;
    const uint32_t slot = ent.y & 0x7ffu, L = ent.y >> 12;
    const bool boxed = (ent.y >> 11) & 1u;
    const uint32_t n = e - s;
    if (n <= kSahSmallNode)
        return sah_node_small(S, A, lo, s, n, depth, slot, L, boxed, lane, warp, left_child, right_child);
    const uint16_t* ord = S.ord[depth & 1u];
    uint16_t* nxt = S.ord[(depth + 1u) & 1u];
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = s + lane; i < e; i += 32) {
        const uint32_t p = ord[i];
        const float4 a = S.lo[p], b = S.hi[p];
        mn[0] = fminf(mn[0], a.x);
        mn[1] = fminf(mn[1], a.y);
        mn[2] = fminf(mn[2], a.z);
        mx[0] = fmaxf(mx[0], b.x);
        mx[1] = fmaxf(mx[1], b.y);
        mx[2] = fmaxf(mx[2], b.z);
        const float c[3] = {a.w, b.w, S.cz[p]};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            cmn[k] = fminf(cmn[k], c[k]);
            cmx[k] = fmaxf(cmx[k], c[k]);
        }
    }
    // Butterfly over the lanes that hold primitives (lanes n..31 hold the
    // identities): ceil(log2(min(n, 32))) steps leave the bounds in lane 0.
    // Leaves need only the box; a split needs the centroid bounds in every lane.
    const uint32_t span = n < 32u ? n : 32u;
    const bool leaf = n <= A.max_leaf;
    if (!boxed)
        for (uint32_t o = 1; o < span; o <<= 1)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
            }
    if (!leaf) {
        float lmn[3] = {cmn[0], cmn[1], cmn[2]}, lmx[3] = {cmx[0], cmx[1], cmx[2]};
        sah_warp_bounds2(lmn, lmx, cmn, cmx);
    }
    const size_t r = 2ull * lo + slot;  // record index
    if (slot == 0 && lane == 0 && !boxed) {  // the subtree root's box, for the top refit
        S.root_lo = make_float4(mn[0], mn[1], mn[2], 0.0f);
        S.root_hi = make_float4(mx[0], mx[1], mx[2], 0.0f);
    }
    if (leaf) {
        if (lane == 0) {
            if (boxed) {
                sah_rec_aux(A.rec, r, lo + s, 0x80000000u | n);
            } else {
                A.rec[2 * r] = make_float4(mn[0], mn[1], mn[2], __uint_as_float(lo + s));
                A.rec[2 * r + 1] = make_float4(mx[0], mx[1], mx[2], __uint_as_float(0x80000000u | n));
            }
            A.rec_l[r] = L;
        }
        for (uint32_t i = s + lane; i < e; i += 32) {
            S.fin[i] = ord[i];
            A.c[lo + i] = i == s ? 1u + L : 0u;
        }
        return 0u;
    }
    // binned SAH over the axes with a centroid extent
    int best_axis = -1, best_split = -1;
    uint32_t best_nl = 0;
    float bscale = 0.0f;
    float lbox[6], rbox[6];
    if (depth < kSahDepthCap) {
        if (n > kSahSmallNode)
            sah_split<16>(S, S.bins[warp], ord, s, e, lane, cmn, cmx, best_axis, best_split, best_nl, bscale, lbox,
                          rbox);
        else
            sah_split<8>(S, S.bins[warp], ord, s, e, lane, cmn, cmx, best_axis, best_split, best_nl, bscale, lbox,
                         rbox);
    }
    uint32_t mid;
    if (best_axis < 0) {
        mid = s + n / 2u;
        for (uint32_t i = s + lane; i < e; i += 32) nxt[i] = ord[i];
    } else {
        mid = s + best_nl;
        const float bmin = sah_pick(cmn, best_axis);
        const uint32_t lt = (1u << lane) - 1u;
        uint32_t nl = 0, nr = 0;
        for (uint32_t b = s; b < e; b += 32) {
            const uint32_t i = b + lane;
            const bool in = i < e;
            const uint32_t p = in ? ord[i] : 0u;
            // the clamp to the last bin cannot move a centroid across a split
            const bool left = in && sah_floor(sah_centroid(S, p, best_axis), bmin, bscale) <= uint32_t(best_split);
            const uint32_t ml = __ballot_sync(0xffffffffu, left), mr = __ballot_sync(0xffffffffu, in && !left);
            if (left)
                nxt[s + nl + __popc(ml & lt)] = uint16_t(p);
            else if (in)
                nxt[mid + nr + __popc(mr & lt)] = uint16_t(p);
            nl += __popc(ml);
            nr += __popc(mr);
        }
    }
    uint32_t cs = 0;
    const bool known = best_axis >= 0;  // the children's boxes are lbox, rbox
    if (lane == 0) {
        if (boxed) {
            sah_rec_aux(A.rec, r, lo + s, lo + mid);
        } else {
            A.rec[2 * r] = make_float4(mn[0], mn[1], mn[2], __uint_as_float(lo + s));
            A.rec[2 * r + 1] = make_float4(mx[0], mx[1], mx[2], __uint_as_float(lo + mid));
        }
        A.rec_l[r] = L;
        cs = atomicAdd(&S.slots, 2u);
        if (known) {
            sah_rec_box(A.rec, 2ull * lo + cs, lbox);
            sah_rec_box(A.rec, 2ull * lo + cs + 1, rbox);
        }
    }
    cs = __shfl_sync(0xffffffffu, cs, 0);
    left_child = sah_entry(s, mid, depth + 1u, cs, L + 1u, known);
    right_child = sah_entry(mid, e, depth + 1u, cs + 1u, 0u, known);
    return 3u;
}

// ---- nodes of more than kSahMax triangles (below the Karras top)
// A persistent launch of blocks of kMidT threads takes them from the node
// queue, one node per block at a time: bounds over the node's range (in the
// order of its depth's parity), 16-bin SAH with one set of bins per warp
// merged before the pricing, a stable partition into the other parity's
// order (each warp counts its slice's left side first), the node's record,
// and its children routed (queue or block list).  A block waits for the next
// entry until it is written, or until every created node is finished (read
// in that order: equal counts mean no node was in progress, and only a node
// in progress creates nodes); every wait is bounded.
constexpr int kMidT = 512;
constexpr int kMidWarps = kMidT / 32;
constexpr uint32_t kMidSpin = 1u << 22;  // polls of a waiting block, at most 1 us apart
constexpr int kMidU = 4;     // positions per thread whose gathers are in flight together
constexpr int kMidBinU = 2;   // the same in the binning pass (its run sums hold 24 registers)
constexpr int kMidPartU = 1;  // and in the partition pass (its children's bounds hold 24)

struct MidArgs {
    const float4* plo;
    const float4* phi;
    const float* pcz;
    uint32_t* ord[2];
    uint4* mq;
    const uint32_t* mready;
    float4* mrec;
    uint32_t* mrec_l;
    SahOut out;
    const int32_t* kl;
    const int32_t* kr;
    const uint32_t* par_in;
    const uint32_t* par_lf;
    float4* box_in;
    float4* box_lf;
    uint32_t* refit_flag;
};

// One thread: entry h of the queue once written (its written flag: 1 without
// bounds, 2 with), or 0 once every created node is finished (or the wait gave
// up: RQ_DERR_QUEUE).
__device__ uint32_t mid_take(const MidArgs& A, uint32_t h) {
    const uint32_t* ctl = A.out.ctl;
    uint32_t nap = 32;
    for (uint32_t it = 0;; ++it) {
        if (h < A.out.mcap) {
            const uint32_t r = rq::ld_acquire(A.mready + h);
            if (r != 0u) return r;
        }
        const uint32_t done = rq::ld_acquire(ctl + 2);
        const uint32_t tail = rq::ld_acquire(ctl + 1);
        if (done == tail) return 0u;
        if (it > kMidSpin) {
            rq::set_err(A.out.err, RQ_DERR_QUEUE);
            return 0u;
        }
        __nanosleep(nap);
        if (nap < 1024u) nap <<= 1;
    }
}

// Bounds accumulators: box min, box max, centroid min, centroid max.
__device__ __forceinline__ void bnd_init(float (&v)[12]) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = INFINITY;
        v[3 + k] = -INFINITY;
        v[6 + k] = INFINITY;
        v[9 + k] = -INFINITY;
    }
}
__device__ __forceinline__ void bnd_add(float (&v)[12], float4 a, float4 b, float cz) {
    v[0] = fminf(v[0], a.x);
    v[1] = fminf(v[1], a.y);
    v[2] = fminf(v[2], a.z);
    v[3] = fmaxf(v[3], b.x);
    v[4] = fmaxf(v[4], b.y);
    v[5] = fmaxf(v[5], b.z);
    v[6] = fminf(v[6], a.w);
    v[7] = fminf(v[7], b.w);
    v[8] = fminf(v[8], cz);
    v[9] = fmaxf(v[9], a.w);
    v[10] = fmaxf(v[10], b.w);
    v[11] = fmaxf(v[11], cz);
}
__device__ __forceinline__ bool bnd_is_min(int k) { return k < 3 || (k >= 6 && k < 9); }

// Block reduction of NV bounds values per thread (sets of 12), into out (shared).
template <int NV>
__device__ __forceinline__ void bnd_reduce(float (&v)[NV], float (*red)[NV], float* out, uint32_t lane, uint32_t warp) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            const float w = __shfl_xor_sync(0xffffffffu, v[k], o);
            v[k] = bnd_is_min(k % 12) ? fminf(v[k], w) : fmaxf(v[k], w);
        }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x < uint32_t(NV)) {
        const uint32_t k = threadIdx.x;
        float x = red[0][k];
        for (uint32_t w = 1; w < uint32_t(kMidWarps); ++w)
            x = bnd_is_min(int(k % 12u)) ? fminf(x, red[w][k]) : fmaxf(x, red[w][k]);
        out[k] = x;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kMidT, 2) k_sah_mid(const MidArgs A) {
    using B16 = SahBinsOf<16>;
    __shared__ alignas(16) uint32_t bins[kMidWarps][B16::words];  // per warp slice
    __shared__ alignas(16) uint32_t mbins[B16::words];             // merged
    __shared__ float red[kMidWarps][24];
    __shared__ float redf[24];
    __shared__ uint32_t part[kMidWarps];
    __shared__ uint4 s_ent[4];
    __shared__ uint32_t s_got;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (;;) {
        if (threadIdx.x == 0) {
            const uint32_t h = atomicAdd(A.out.ctl, 1u);
            const uint32_t r = mid_take(A, h);
            s_got = r;
            if (r != 0u) {
                const uint4* q = A.mq + 4 * size_t(h);
                s_ent[0] = __ldcg(q);
                if (r == 2u) {
                    s_ent[1] = __ldcg(q + 1);
                    s_ent[2] = __ldcg(q + 2);
                    s_ent[3] = __ldcg(q + 3);
                }
            }
        }
        __syncthreads();
        const uint32_t got = s_got;
        if (got == 0u) break;
        const uint4 hdr = s_ent[0];
        const uint32_t s = hdr.x, e = hdr.y, depth = hdr.z & 0xffu, L = hdr.z >> 8, rn = hdr.w;
        const uint32_t n = e - s;
        const uint32_t* in = A.ord[depth & 1u];
        uint32_t* out = A.ord[(depth + 1u) & 1u];
        // the node's bounds: from its entry, or (a SAH root) over its range
        if (got == 2u) {
            if (threadIdx.x < 12u) redf[threadIdx.x] = __uint_as_float((&s_ent[1].x)[threadIdx.x]);
            __syncthreads();
        } else {
            float v[12];
            bnd_init(v);
            for (uint32_t i0 = s + threadIdx.x; i0 < e; i0 += kMidT * kMidU) {
                uint32_t p[kMidU];
#pragma unroll
                for (int u = 0; u < kMidU; ++u) {
                    const uint32_t i = i0 + uint32_t(u) * kMidT;
                    p[u] = i < e ? __ldcg(in + i) : kSahNone;
                }
#pragma unroll
                for (int u = 0; u < kMidU; ++u) {
                    const uint32_t q = p[u] != kSahNone ? p[u] : 0u;  // position 0 exists (n > kSahMax)
                    const float4 a = __ldg(A.plo + q), b = __ldg(A.phi + q);
                    const float cz = __ldg(A.pcz + q);
                    if (p[u] != kSahNone) bnd_add(v, a, b, cz);
                }
            }
            bnd_reduce<12>(v, reinterpret_cast<float (*)[12]>(&red[0][0]), redf, lane, warp);
        }
        float mn[3], mx[3], cmn[3], cmx[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = redf[k];
            mx[k] = redf[3 + k];
            cmn[k] = redf[6 + k];
            cmx[k] = redf[9 + k];
        }
        __syncthreads();  // redf is reused below
        // warp slices of a multiple of 32 positions, in order: the same slices
        // are binned and partitioned, so a warp's left count is in its bins
        const uint32_t q32 = ((n + 32u * kMidWarps - 1u) / (32u * kMidWarps)) * 32u;
        const uint32_t ws = s + min(n, warp * q32), we = s + min(n, (warp + 1u) * q32);
        int best_axis = -1, best_split = -1;
        uint32_t best_nl = 0;
        float scale[3] = {0.0f, 0.0f, 0.0f};
        if (depth < kSahDepthCap) {
            sah_scales<16>(cmn, cmx, scale, lane);
            sah_bins_clear<16>(bins[warp], lane);
            __syncwarp();
            // Each lane a run of consecutive positions, kMidBinU of them in
            // flight at a time.  Consecutive triangles mostly share a bin, so
            // a lane sums its current bin per axis in registers and adds it to
            // the warp's bins only when the bin changes (and at the end): min
            // and max of the partial boxes are exact, so the bins are the same.
            const uint32_t run = ((we - ws + 31u) >> 5) | 1u;
            const uint32_t r0 = ws + lane * run, r1 = min(we, r0 + run);
            constexpr uint32_t F = B16::slots;
            uint32_t cb[3] = {kSahNone, kSahNone, kSahNone}, cn[3] = {0u, 0u, 0u};
            float bl[3][3], bh[3][3];
            auto flush = [&](int k) {
                uint32_t* bn = bins[warp] + k * 16 + cb[k];
                atomicAdd(bn, cn[k]);
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    atomicMin(bn + (1 + q) * F, rq::f2o(bl[k][q]));
                    atomicMax(bn + (4 + q) * F, rq::f2o(bh[k][q]));
                }
            };
            for (uint32_t i0 = r0; i0 < r1; i0 += kMidBinU) {
                uint32_t p[kMidBinU];
#pragma unroll
                for (int u = 0; u < kMidBinU; ++u) {
                    const uint32_t i = i0 + uint32_t(u);
                    p[u] = i < r1 ? __ldcg(in + i) : kSahNone;
                }
                float4 a4[kMidBinU], b4[kMidBinU];
                float cz[kMidBinU];
#pragma unroll
                for (int u = 0; u < kMidBinU; ++u) {
                    const uint32_t q = p[u] != kSahNone ? p[u] : 0u;
                    a4[u] = __ldg(A.plo + q);
                    b4[u] = __ldg(A.phi + q);
                    cz[u] = __ldg(A.pcz + q);
                }
#pragma unroll
                for (int u = 0; u < kMidBinU; ++u) {
                    if (p[u] == kSahNone) continue;
                    const float c[3] = {a4[u].w, b4[u].w, cz[u]};
                    const float lo3[3] = {a4[u].x, a4[u].y, a4[u].z}, hi3[3] = {b4[u].x, b4[u].y, b4[u].z};
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        if (!(scale[k] > 0.0f)) continue;
                        const uint32_t bin = sah_bin<16>(c[k], cmn[k], scale[k]);
                        if (bin != cb[k]) {
                            if (cb[k] != kSahNone) flush(k);
                            cb[k] = bin;
                            cn[k] = 0u;
#pragma unroll
                            for (int q = 0; q < 3; ++q) {
                                bl[k][q] = INFINITY;
                                bh[k][q] = -INFINITY;
                            }
                        }
                        ++cn[k];
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            bl[k][q] = fminf(bl[k][q], lo3[q]);
                            bh[k][q] = fmaxf(bh[k][q], hi3[q]);
                        }
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (cb[k] != kSahNone) flush(k);
            __syncthreads();
            for (uint32_t w = threadIdx.x; w < B16::words; w += kMidT) {
                const uint32_t f = w / B16::slots;
                uint32_t x = bins[0][w];
                for (uint32_t c = 1; c < uint32_t(kMidWarps); ++c) {
                    const uint32_t y = bins[c][w];
                    x = f == 0 ? x + y : (f <= 3 ? min(x, y) : max(x, y));
                }
                mbins[w] = x;
            }
            __syncthreads();
            float lbx[6], rbx[6];  // not needed: the partition pass sums the children's bounds
            sah_choose<16>(mbins, scale, lane, best_axis, best_split, best_nl, lbx, rbx);  // every warp, the same result
        }
        // the stable partition, and both children's bounds
        uint32_t mid;
        float cv[24];
        bnd_init(*reinterpret_cast<float (*)[12]>(&cv[0]));
        bnd_init(*reinterpret_cast<float (*)[12]>(&cv[12]));
        if (best_axis < 0) {
            mid = s + n / 2u;
            for (uint32_t i = s + threadIdx.x; i < e; i += kMidT) {
                const uint32_t p = __ldcg(in + i);
                out[i] = p;
                const float4 a = __ldg(A.plo + p), b = __ldg(A.phi + p);
                bnd_add(*reinterpret_cast<float (*)[12]>(&cv[i < mid ? 0 : 12]), a, b, __ldg(A.pcz + p));
            }
        } else {
            mid = s + best_nl;
            const float bmin = sah_pick(cmn, best_axis), bscale = sah_pick(scale, best_axis);
            // this warp's left count: its slice's bins up to the split on the axis
            {
                const uint32_t* bw = bins[warp] + best_axis * 16;
                const uint32_t cnt = lane < 16u && lane <= uint32_t(best_split) ? bw[lane] : 0u;
                const uint32_t nl = __reduce_add_sync(0xffffffffu, cnt);
                if (lane == 0) part[warp] = nl;
            }
            __syncthreads();
            uint32_t offl = 0, offr = 0;
            for (uint32_t w = 0; w < warp; ++w) {
                const uint32_t len = min(n, (w + 1u) * q32) - min(n, w * q32);
                offl += part[w];
                offr += len - part[w];
            }
            const uint32_t lt = (1u << lane) - 1u;
            for (uint32_t b = ws; b < we; b += 32u * kMidPartU) {
                uint32_t p[kMidPartU];
#pragma unroll
                for (int u = 0; u < kMidPartU; ++u) {
                    const uint32_t i = b + uint32_t(u) * 32u + lane;
                    p[u] = i < we ? __ldcg(in + i) : kSahNone;
                }
                float4 a4[kMidPartU], b4[kMidPartU];
                float cz[kMidPartU];
#pragma unroll
                for (int u = 0; u < kMidPartU; ++u) {
                    const uint32_t q = p[u] != kSahNone ? p[u] : 0u;
                    a4[u] = __ldg(A.plo + q);
                    b4[u] = __ldg(A.phi + q);
                    cz[u] = __ldg(A.pcz + q);
                }
#pragma unroll
                for (int u = 0; u < kMidPartU; ++u) {
                    const bool in_range = p[u] != kSahNone;
                    const float c = best_axis == 0 ? a4[u].w : (best_axis == 1 ? b4[u].w : cz[u]);
                    const bool left = in_range && sah_floor(c, bmin, bscale) <= uint32_t(best_split);
                    const uint32_t ml = __ballot_sync(0xffffffffu, left),
                                   mr = __ballot_sync(0xffffffffu, in_range && !left);
                    if (left) {
                        out[s + offl + __popc(ml & lt)] = p[u];
                        bnd_add(*reinterpret_cast<float (*)[12]>(&cv[0]), a4[u], b4[u], cz[u]);
                    } else if (in_range) {
                        out[mid + offr + __popc(mr & lt)] = p[u];
                        bnd_add(*reinterpret_cast<float (*)[12]>(&cv[12]), a4[u], b4[u], cz[u]);
                    }
                    offl += __popc(ml);
                    offr += __popc(mr);
                }
            }
        }
        __threadfence();  // the new order before the children are published
        bnd_reduce<24>(cv, red, redf, lane, warp);
        if (threadIdx.x == 0) {
            const uint32_t k = atomicAdd(A.out.ctl + 3, 1u);
            if (k < A.out.mcap) {
                A.mrec[2 * size_t(k)] = make_float4(mn[0], mn[1], mn[2], __uint_as_float(s));
                A.mrec[2 * size_t(k) + 1] = make_float4(mx[0], mx[1], mx[2], __uint_as_float(mid));
                A.mrec_l[k] = L;
            } else {
                rq::set_err(A.out.err, RQ_DERR_QUEUE);
            }
            float lb[12], rb[12];
#pragma unroll
            for (int k2 = 0; k2 < 12; ++k2) {
                lb[k2] = redf[k2];
                rb[k2] = redf[12 + k2];
            }
            sah_route(A.out, s, mid, depth + 1u, L + 1u, kSahNone, lb);
            sah_route(A.out, mid, e, depth + 1u, 0u, kSahNone, rb);
            if (rn != kSahNone)
                sah_refit_up(rn, make_float4(mn[0], mn[1], mn[2], 0.0f), make_float4(mx[0], mx[1], mx[2], 0.0f), A.kl,
                             A.kr, A.par_in, A.par_lf, A.box_in, A.box_lf, A.refit_flag, A.out.err);
            __threadfence();
            atomicAdd(A.out.ctl + 2, 1u);  // finished, after its children were created
        }
        __syncthreads();
    }
}

// One block per subtree of at most kSahMax triangles (taken from a counter):
// load its primitives in the order and at the depth it was handed over, build
// it level by level (a warp per node), write its leaf-ordered triangles, mark
// its unused record slots, then, under a Karras node, refit the Karras nodes
// above it.
__global__ void __launch_bounds__(kSahT, 3) k_sah_build(const SahArgs A) {
    extern __shared__ __align__(16) unsigned char s_raw[];
    SahShared& S = *reinterpret_cast<SahShared*>(s_raw);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t nsubtrees = *A.count;
    for (;;) {
        if (threadIdx.x == 0) S.job = atomicAdd(A.next, 1u);
        __syncthreads();
        const uint32_t j = S.job;
        if (j >= nsubtrees) break;
        const uint32_t lo = A.list[j];
        const uint32_t nsub = A.shi[lo] - lo + 1u;
        // depth below the SAH root and starting order: from the node queue's
        // partitions (k_sah_mid) or, under a Karras node, 0 and the Morton order.
        // Slot i holds the primitive at position i of that order (a sorted
        // position anywhere in the parent's range, after a partition).
        const uint32_t d0 = A.sdepth[lo];
        const uint32_t* g = A.ord[d0 & 1u];
        for (uint32_t i = threadIdx.x; i < nsub; i += kSahT) {
            const uint32_t p = __ldcg(g + lo + i);
            S.lo[i] = __ldg(A.plo + p);
            S.hi[i] = __ldg(A.phi + p);
            S.cz[i] = __ldg(A.pcz + p);
            S.id[i] = A.sids[p];
            S.ord[d0 & 1u][i] = uint16_t(i);
        }
        if (threadIdx.x == 0) {
            S.cnt[0] = 1u;
            S.cnt[1] = 0u;
            S.slots = 1u;
            S.list[0][0] = sah_entry(0u, nsub, d0, 0u, A.sL[lo]);
        }
        __syncthreads();
        // Level by level, a warp per node; a node at depth d reads the leaf
        // order at parity d and writes its partition to parity d + 1.
        int cur = 0;
        for (uint32_t guard = 0;; ++guard) {
            const uint32_t m = S.cnt[cur];
            if (m == 0u || guard > 64u) break;
            for (uint32_t k = warp; k < m; k += kSahWarps) {
                uint2 lc, rc;
                const uint32_t push = sah_node(S, A, lo, S.list[cur][k], lane, warp, lc, rc);
                if (push && lane == 0) {
                    uint32_t b = atomicAdd(&S.cnt[cur ^ 1], uint32_t(__popc(push)));
                    if (push & 1u) S.list[cur ^ 1][b++] = lc;
                    if (push & 2u) S.list[cur ^ 1][b] = rc;
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) S.cnt[cur] = 0u;
            cur ^= 1;
            __syncthreads();
        }
        // The leaf-ordered triangles, permutation and keys of the whole subtree
        // by the whole block (every leaf recorded its range of the final order):
        // the index and vertex fetches of all its triangles are in flight
        // together instead of a leaf's few at a time.
        for (uint32_t i = threadIdx.x; i < nsub; i += kSahT) {
            const uint32_t k = lo + i, gid = S.id[S.fin[i]];
            rq::F3 p0, p1, p2;
            rq::load_tri(A.pos, A.sf, A.idx, gid, p0, p1, p2);
            float4* tp = reinterpret_cast<float4*>(A.tris + k);
            tp[0] = make_float4(p0.x, p0.y, p0.z, 0.0f);
            tp[1] = make_float4(p1.x, p1.y, p1.z, 0.0f);
            tp[2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
            A.perm[k] = gid;
            A.keys_out[k] = A.skeys[k];
        }
        for (uint32_t k = S.slots + threadIdx.x; k < 2u * nsub; k += kSahT) A.rec_l[2ull * lo + k] = kNoRecord;
        if (threadIdx.x == 0 && A.snode[lo] != kSahNone)
            sah_refit_up(A.snode[lo], S.root_lo, S.root_hi, A.kl, A.kr, A.par_in, A.par_lf, A.box_in, A.box_lf,
                         A.refit_flag, A.err);
        __syncthreads();
    }
}

// Node writes: every record (the block subtrees' and the node queue's) at
// A[first] + L (left child next to it, right child at A[its first position];
// leaves as ~first / count), every Karras node above the SAH roots (more
// than K primitives) likewise from its Karras range and refitted box.
// One node record (box, first position in w; box, the right child's first
// position or bit 31 | the leaf count in w) at its pre-order position.
__device__ __forceinline__ void sah_emit_record(float4 a, float4 b, uint32_t L, const uint32_t* __restrict__ A,
                                                rq_bvh2_node* __restrict__ out) {
    const uint32_t first = __float_as_uint(a.w), aux = __float_as_uint(b.w);
    const uint32_t pre = A[first] + L;
    const bool leaf = (aux >> 31) != 0u;
    const int32_t lc = leaf ? ~int32_t(first) : int32_t(pre + 1u);
    const int32_t rc = leaf ? int32_t(aux & 0x7fffffffu) : int32_t(A[aux]);
    float4* o = reinterpret_cast<float4*>(out + pre);
    o[0] = make_float4(a.x, a.y, a.z, __int_as_float(lc));
    o[1] = make_float4(b.x, b.y, b.z, __int_as_float(rc));
}

__global__ void __launch_bounds__(kT) k_sah_emit(uint32_t n, uint32_t K, uint32_t max_leaf,
                                                 const float4* __restrict__ rec, const uint32_t* __restrict__ rec_l,
                                                 const float4* __restrict__ mrec, const uint32_t* __restrict__ mrec_l,
                                                 const uint32_t* __restrict__ mcount, uint32_t mcap,
                                                 const int32_t* __restrict__ kr, const uint32_t* __restrict__ klo,
                                                 const uint32_t* __restrict__ khi,
                                                 const uint32_t* __restrict__ par_in, const float4* box_in,
                                                 const uint32_t* __restrict__ c, const uint32_t* __restrict__ A,
                                                 rq_bvh2_node* __restrict__ out, uint32_t* __restrict__ counts) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < 2u * n; i += gridDim.x * kT) {
        const uint32_t L = rec_l[i];
        if (L == kNoRecord) continue;
        sah_emit_record(rec[2 * size_t(i)], rec[2 * size_t(i) + 1], L, A, out);
    }
    const uint32_t m = min(*mcount, mcap);
    for (uint32_t k = blockIdx.x * kT + threadIdx.x; k < m; k += gridDim.x * kT)
        sah_emit_record(mrec[2 * size_t(k)], mrec[2 * size_t(k) + 1], mrec_l[k], A, out);
    for (uint32_t p = blockIdx.x * kT + threadIdx.x; p + 1u < n; p += gridDim.x * kT) {
        if (rq::count_in(klo, khi, p) <= K) continue;
        uint32_t L = 0, par = par_in[p];
        while (par != rq::kNoParent && (par & 1u) == 0u) {
            ++L;
            par = par_in[par >> 1];
        }
        const uint32_t pre = A[klo[p]] + L;
        const int32_t r = kr[p];
        const uint32_t rlo = r < 0 ? (uint32_t(r) & 0x7fffffffu) : klo[r];
        const float4 lo = rq::ld_cg4(box_in + 2 * size_t(p)), hi = rq::ld_cg4(box_in + 2 * size_t(p) + 1);
        float4* o = reinterpret_cast<float4*>(out + pre);
        o[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(int32_t(pre + 1u)));
        o[1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(int32_t(A[rlo])));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        counts[0] = A[n - 1u] + c[n - 1u];
        counts[3] = max_leaf;
    }
}

// ------------------------------------------------------------------ refit
// Parent links of an emitted binary BVH (any layout with the root at 0).
__global__ void __launch_bounds__(kT) k_parents2(const rq_bvh2_node* __restrict__ nodes, const uint32_t* counts,
                                                 uint32_t* __restrict__ parent, uint32_t* __restrict__ flag) {
    const uint32_t n2 = counts[0];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n2; i += gridDim.x * kT) {
        const rq_bvh2_node nd = nodes[i];
        flag[i] = 0u;
        if (i == 0) parent[0] = rq::kNoParent;
        if (nd.left_child >= 0) {
            parent[nd.left_child] = i;
            parent[nd.right_child] = i;
        }
    }
}

// Leaves: new triangle copies from the moved vertices, leaf boxes, then the
// atomic walk to the root recomputing inner boxes.
__global__ void __launch_bounds__(kT) k_refit2(const float* __restrict__ pos, uint32_t sf,
                                               const uint32_t* __restrict__ idx, const uint32_t* counts,
                                               const uint32_t* __restrict__ perm, rq_bvh2_node* nodes,
                                               rq_triangle* __restrict__ tris, const uint32_t* __restrict__ parent,
                                               uint32_t* flag, uint32_t* err) {
    const uint32_t n2 = counts[0];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n2; i += gridDim.x * kT) {
        const rq_bvh2_node nd = nodes[i];
        if (nd.left_child >= 0) continue;
        const uint32_t first = uint32_t(~nd.left_child), cnt = uint32_t(nd.right_child);
        float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t q = first; q < first + cnt; ++q) {
            rq::F3 p0, p1, p2;
            rq::load_tri(pos, sf, idx, perm[q], p0, p1, p2);
            float4* tp = reinterpret_cast<float4*>(tris + q);
            tp[0] = make_float4(p0.x, p0.y, p0.z, 0.0f);
            tp[1] = make_float4(p1.x, p1.y, p1.z, 0.0f);
            tp[2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
            mn[0] = fminf(mn[0], fminf(p0.x, fminf(p1.x, p2.x)));
            mn[1] = fminf(mn[1], fminf(p0.y, fminf(p1.y, p2.y)));
            mn[2] = fminf(mn[2], fminf(p0.z, fminf(p1.z, p2.z)));
            mx[0] = fmaxf(mx[0], fmaxf(p0.x, fmaxf(p1.x, p2.x)));
            mx[1] = fmaxf(mx[1], fmaxf(p0.y, fmaxf(p1.y, p2.y)));
            mx[2] = fmaxf(mx[2], fmaxf(p0.z, fmaxf(p1.z, p2.z)));
        }
        float4* o = reinterpret_cast<float4*>(nodes + i);
        __stcg(o, make_float4(mn[0], mn[1], mn[2], __int_as_float(nd.left_child)));
        __stcg(o + 1, make_float4(mx[0], mx[1], mx[2], __int_as_float(nd.right_child)));
        uint32_t p = parent[i];
        uint32_t guard = 0;
        while (p != rq::kNoParent) {
            // publishes this thread's last box; the second arrival sees the sibling's
            if (rq::atom_add_acq_rel(&flag[p], 1u) == 0u) break;
            const float4* pn = reinterpret_cast<const float4*>(nodes + p);
            const float4 pa = rq::ld_cg4(pn), pb = rq::ld_cg4(pn + 1);
            const int32_t l = __float_as_int(pa.w), r = __float_as_int(pb.w);
            const float4* ln = reinterpret_cast<const float4*>(nodes + l);
            const float4* rn = reinterpret_cast<const float4*>(nodes + r);
            const float4 la = rq::ld_cg4(ln), lb = rq::ld_cg4(ln + 1), ra = rq::ld_cg4(rn), rb = rq::ld_cg4(rn + 1);
            __stcg(reinterpret_cast<float4*>(nodes + p),
                   make_float4(fminf(la.x, ra.x), fminf(la.y, ra.y), fminf(la.z, ra.z), pa.w));
            __stcg(reinterpret_cast<float4*>(nodes + p) + 1,
                   make_float4(fmaxf(lb.x, rb.x), fmaxf(lb.y, rb.y), fmaxf(lb.z, rb.z), pb.w));
            p = parent[p];
            if (++guard > 256u) {
                rq::set_err(err, RQ_DERR_REFIT);
                break;
            }
        }
    }
}

// 4-wide boxes from the refitted binary nodes through the slot map written
// by the collapse.
__global__ void __launch_bounds__(kT) k_refit4(const rq_bvh2_node* __restrict__ n2, const uint32_t* counts,
                                               const int32_t* __restrict__ map4, rq_bvh4_node* __restrict__ n4) {
    const uint32_t m = counts[1];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < 4 * m; i += gridDim.x * kT) {
        const int32_t s = map4[i];
        if (s < 0) continue;
        const uint32_t node = i >> 2, k = i & 3u;
        const rq_bvh2_node c = n2[s];
        n4[node].min_x[k] = c.aabb_min[0];
        n4[node].max_x[k] = c.aabb_max[0];
        n4[node].min_y[k] = c.aabb_min[1];
        n4[node].max_y[k] = c.aabb_max[1];
        n4[node].min_z[k] = c.aabb_min[2];
        n4[node].max_z[k] = c.aabb_max[2];
    }
}

inline uint32_t grid_for(uint32_t n, int sms) {
    const uint32_t b = (n + kT - 1) / kT;
    const uint32_t cap = uint32_t(sms) * 8u;
    return std::max(1u, std::min(b, cap));
}

}  // namespace

size_t rq_build_scratch_carve(void* base, uint32_t n, BuildScratch& s, bool sah) {
    Carve c{reinterpret_cast<uintptr_t>(base), 0};
    const size_t N = n ? n : 1;
    const uint32_t tiles = rq_sort_tiles(uint32_t(N)), stiles = rq_scan_tiles(uint32_t(N));
    s.cent = c.take<float4>(N);
    s.bounds = c.take<uint32_t>(8);
    s.keys[0] = c.take<uint32_t>(N);
    s.vals[0] = c.take<uint32_t>(N);
    s.keys[1] = c.take<uint32_t>(N);
    s.vals[1] = c.take<uint32_t>(N);
    s.hist = c.take<uint32_t>(4 * 256);
    s.sort_status = c.take<uint32_t>(4ull * tiles * 256);
    s.tile_ctr = c.take<uint32_t>(16);
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
    s.scan_status = c.take<uint32_t>(stiles + 1);
    s.q = c.take<uint32_t>(N);
    s.cand = c.take<int32_t>(4 * N);
    s.child_q = c.take<int32_t>(4 * N);
    s.sz = c.take<uint32_t>(N);
    s.cpar = c.take<uint32_t>(N);
    s.cacc = c.take<unsigned long long>(N);
    s.coll_ctl = c.take<uint32_t>(256);
    s.sah_hi = s.sah_L = s.sah_node = s.sah_list = s.sah_depth = s.sah_rec_l = nullptr;
    s.sah_rec = s.sah_plo = s.sah_phi = s.sah_mrec = nullptr;
    s.sah_pcz = nullptr;
    s.sah_ord[0] = s.sah_ord[1] = s.sah_mready = s.sah_mrec_l = s.sah_ctl = nullptr;
    s.sah_mq = nullptr;
    s.sah_mcap = 0;
    if (sah) {
        s.sah_hi = c.take<uint32_t>(N);
        s.sah_L = c.take<uint32_t>(N);
        s.sah_node = c.take<uint32_t>(N);
        s.sah_list = c.take<uint32_t>(N);
        s.sah_depth = c.take<uint32_t>(N);
        s.sah_rec = c.take<float4>(4 * N);
        s.sah_rec_l = c.take<uint32_t>(2 * N);
        s.sah_plo = c.take<float4>(N);
        s.sah_phi = c.take<float4>(N);
        s.sah_pcz = c.take<float>(N);
        s.sah_ord[0] = c.take<uint32_t>(N);
        s.sah_ord[1] = c.take<uint32_t>(N);
        // nodes of more than kSahMax triangles: those at one depth hold disjoint
        // ranges of more than kSahMax positions (at most N / kSahMax of them),
        // and they lie at most kSahDepthCap + 6 deep (SAH splits to the depth
        // cap, then halvings from at most RQ_SAH_SUBTREE_MAX <= 64 x kSahMax down)
        s.sah_mcap = uint32_t(kSahMidDepths * (N / kSahMax) + 64);
        s.sah_mq = c.take<uint4>(4 * size_t(s.sah_mcap));
        s.sah_mready = c.take<uint32_t>(s.sah_mcap);
        s.sah_mrec = c.take<float4>(2 * size_t(s.sah_mcap));
        s.sah_mrec_l = c.take<uint32_t>(s.sah_mcap);
        s.sah_ctl = c.take<uint32_t>(16);
    }
    return c.off + 256;
}

namespace {

// Per-position boxes, the SAH roots, the nodes of more than kSahMax triangles
// (node queue), the block subtrees (with the top refit), the scan of the
// emission counts and the node writes.
int launch_sah(rq_ctx* ctx, rq_bvh* bvh, BuildScratch& s, const float* pos, uint32_t sf, const uint32_t* idx,
               uint32_t n, uint32_t max_leaf, uint32_t K, const uint32_t* skeys, const uint32_t* sids,
               cudaStream_t st) {
    const int sms = ctx->num_sms;
    static const size_t kSmem = sizeof(SahShared);
    static int per_sm = [] {
        cudaFuncSetAttribute(k_sah_build, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmem));
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sah_build, kSahT, kSmem);
        return b > 0 ? b : 1;
    }();
    static int mid_per_sm = [] {
        int b = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_sah_mid, kMidT, 0);
        return b > 0 ? b : 1;
    }();
    // queue counters and written flags; the block list's count is tile_ctr[13]
    // (zeroed with the build's counters)
    cudaError_t e = cudaMemsetAsync(s.sah_ctl, 0, 16 * sizeof(uint32_t), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.sah_mready, 0, sizeof(uint32_t) * s.sah_mcap, st);
    k_sah_pbox<<<grid_for(n, sms), kT, 0, st>>>(pos, sf, idx, n, sids, s.cent, s.sah_plo, s.sah_phi, s.sah_pcz,
                                                s.sah_ord[0]);
    SahOut o;
    o.list = s.sah_list;
    o.count = s.tile_ctr + 13;
    o.shi = s.sah_hi;
    o.sL = s.sah_L;
    o.sdepth = s.sah_depth;
    o.snode = s.sah_node;
    o.mq = s.sah_mq;
    o.mready = s.sah_mready;
    o.mcap = s.sah_mcap;
    o.ctl = s.sah_ctl;
    o.err = ctx->d_err;
    k_sah_roots<<<grid_for(n, sms), kT, 0, st>>>(n, K, s.kl, s.kr, s.klo, s.khi, s.par_in, o);
    MidArgs m;
    m.plo = s.sah_plo;
    m.phi = s.sah_phi;
    m.pcz = s.sah_pcz;
    m.ord[0] = s.sah_ord[0];
    m.ord[1] = s.sah_ord[1];
    m.mq = s.sah_mq;
    m.mready = s.sah_mready;
    m.mrec = s.sah_mrec;
    m.mrec_l = s.sah_mrec_l;
    m.out = o;
    m.kl = s.kl;
    m.kr = s.kr;
    m.par_in = s.par_in;
    m.par_lf = s.par_lf;
    m.box_in = s.box_in;
    m.box_lf = s.box_lf;
    m.refit_flag = s.refit_flag;
    if (n > kSahMax) k_sah_mid<<<uint32_t(sms) * uint32_t(mid_per_sm), kMidT, 0, st>>>(m);
    SahArgs a;
    a.n = n;
    a.max_leaf = max_leaf;
    a.plo = s.sah_plo;
    a.phi = s.sah_phi;
    a.pcz = s.sah_pcz;
    a.ord[0] = s.sah_ord[0];
    a.ord[1] = s.sah_ord[1];
    a.sdepth = s.sah_depth;
    a.pos = pos;
    a.sf = sf;
    a.idx = idx;
    a.skeys = skeys;
    a.sids = sids;
    a.kl = s.kl;
    a.kr = s.kr;
    a.par_in = s.par_in;
    a.par_lf = s.par_lf;
    a.box_in = s.box_in;
    a.box_lf = s.box_lf;
    a.refit_flag = s.refit_flag;
    a.shi = s.sah_hi;
    a.sL = s.sah_L;
    a.snode = s.sah_node;
    a.list = s.sah_list;
    a.count = s.tile_ctr + 13;
    a.next = s.tile_ctr + 12;
    a.rec = s.sah_rec;
    a.rec_l = s.sah_rec_l;
    a.c = s.c;
    a.tris = bvh->tris;
    a.perm = bvh->perm;
    a.keys_out = bvh->skeys;
    a.err = ctx->d_err;
    k_sah_build<<<uint32_t(sms) * uint32_t(per_sm), kSahT, kSmem, st>>>(a);
    if (e == cudaSuccess) e = cudaMemsetAsync(s.tile_ctr + 8, 0, sizeof(uint32_t), st);
    rq_launch_scan(ctx, s.c, s.a, n, s.scan_status, s.tile_ctr + 8, st);
    k_sah_emit<<<grid_for(2 * n, sms), kT, 0, st>>>(n, K, max_leaf, s.sah_rec, s.sah_rec_l, s.sah_mrec, s.sah_mrec_l,
                                                    s.sah_ctl + 3, s.sah_mcap, s.kr, s.klo, s.khi, s.par_in,
                                                    s.box_in, s.c, s.a, bvh->nodes2, bvh->d_counts);
    return rq_cuda_status(ctx, e == cudaSuccess ? cudaGetLastError() : e, "SAH-subtree build launch");
}

}  // namespace

int rq_launch_build(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                    uint32_t n, uint32_t max_leaf, bool collapse, cudaStream_t st, uint32_t sah_max) {
    BuildScratch s;
    const bool sah = sah_max > 0;
    if (sah && (sah_max > RQ_SAH_SUBTREE_MAX || sah_max < max_leaf))
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "SAH subtree size out of range");
    const size_t need = rq_build_scratch_carve(nullptr, n, s, sah);
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    rq_build_scratch_carve(ctx->scratch, n, s, sah);
    const uint32_t sf = stride_bytes / 4;
    const int sms = ctx->num_sms;

    // bounds: min = 0xffffffff (ordered +inf side), max = 0
    cudaMemsetAsync(s.bounds, 0xff, 3 * sizeof(uint32_t), st);
    cudaMemsetAsync(s.bounds + 3, 0x00, 3 * sizeof(uint32_t), st);
    cudaMemsetAsync(s.tile_ctr, 0, 16 * sizeof(uint32_t), st);
    if (n > 1) cudaMemsetAsync(s.refit_flag, 0, sizeof(uint32_t) * (n - 1), st);

    k_centroids<<<grid_for(n, sms), kT, 0, st>>>(pos, sf, idx, n, s.cent, s.bounds);
    k_morton<<<grid_for(n, sms), kT, 0, st>>>(s.cent, n, s.bounds, s.keys[0], s.vals[0]);
    int rb = 0;
    rc = rq_launch_sort(ctx, s, n, 30, st, &rb);
    if (rc) return rc;
    const uint32_t* skeys = s.keys[rb];
    const uint32_t* sids = s.vals[rb];
    k_karras<<<grid_for(n, sms), kT, 0, st>>>(skeys, n, s.kl, s.kr, s.klo, s.khi, s.par_in, s.par_lf);
    if (sah) {
        rc = launch_sah(ctx, bvh, s, pos, sf, idx, n, max_leaf, sah_max, skeys, sids, st);
        if (rc) return rc;
        if (collapse) return rq_launch_collapse(ctx, bvh, s, st);
        return RQ_OK;
    }
    // the handed-over walks: listed in the centroid array (free after the
    // Morton codes), counted in tile_ctr[12] (zeroed above, unused by the sort)
    uint32_t* top_list = reinterpret_cast<uint32_t*>(s.cent);
    uint32_t* top_cnt = s.tile_ctr + 12;
    k_leaves_local<<<(n + kLocal - 1) / kLocal, kT, 0, st>>>(pos, sf, idx, n, max_leaf, skeys, sids, s.kl, s.kr,
                                                             s.klo, s.khi, s.par_in, s.par_lf, s.box_in, s.box_lf,
                                                             s.refit_flag, s.c, bvh->tris, bvh->perm, bvh->skeys,
                                                             top_list, top_cnt, ctx->d_err);
    k_refit_top<<<uint32_t(sms) * 4u, kT, 0, st>>>(s.kl, s.kr, s.par_in, s.box_in, s.box_lf, s.refit_flag, top_list,
                                                   top_cnt, ctx->d_err);
    rq_launch_scan(ctx, s.c, s.a, n, s.scan_status, s.tile_ctr + 8, st);
    k_emit2<<<grid_for(n, sms), kT, 0, st>>>(n, max_leaf, s.kr, s.klo, s.khi, s.par_in, s.par_lf, s.box_in, s.box_lf,
                                             s.c, s.a, bvh->nodes2, bvh->d_counts);
    rc = rq_cuda_status(ctx, cudaGetLastError(), "build launch");
    if (rc) return rc;
    if (collapse) return rq_launch_collapse(ctx, bvh, s, st);
    return RQ_OK;
}

int rq_launch_refit(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                    cudaStream_t st) {
    const uint32_t n2cap = bvh->cap_nodes2;
    const size_t need = sizeof(uint32_t) * (2ull * n2cap + 64);
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    uint32_t* parent = static_cast<uint32_t*>(ctx->scratch);
    uint32_t* flag = parent + n2cap + 32;
    const int sms = ctx->num_sms;
    k_parents2<<<grid_for(n2cap, sms), kT, 0, st>>>(bvh->nodes2, bvh->d_counts, parent, flag);
    k_refit2<<<grid_for(n2cap, sms), kT, 0, st>>>(pos, stride_bytes / 4, idx, bvh->d_counts, bvh->perm, bvh->nodes2,
                                                  bvh->tris, parent, flag, ctx->d_err);
    if (bvh->has4) {
        k_refit4<<<grid_for(4 * bvh->cap_nodes4, sms), kT, 0, st>>>(bvh->nodes2, bvh->d_counts, bvh->map4,
                                                                    bvh->nodes4);
    }
    return rq_cuda_status(ctx, cudaGetLastError(), "refit launch");
}
