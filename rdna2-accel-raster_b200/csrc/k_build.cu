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
// memory once for the emission.  Only nodes whose range crosses a block
// boundary (a few per block and level) use the device-scope acquire-release
// count of refit_walk.  Unions are exact, so the boxes equal refit_walk's.
constexpr uint32_t kLocal = 256;  // 17 KB of shared memory per block (measured: faster than 512)

__global__ void __launch_bounds__(kT) k_leaves_local(
    const float* __restrict__ pos, uint32_t sf, const uint32_t* __restrict__ idx, uint32_t n, uint32_t max_leaf,
    const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ sids, const int32_t* __restrict__ kl,
    const int32_t* __restrict__ kr, const uint32_t* __restrict__ klo, const uint32_t* __restrict__ khi,
    const uint32_t* __restrict__ par_in, const uint32_t* __restrict__ par_lf, float4* box_in,
    float4* __restrict__ box_lf, uint32_t* refit_flag, uint32_t* __restrict__ c_out, rq_triangle* __restrict__ tris,
    uint32_t* __restrict__ perm, uint32_t* __restrict__ keys_out, uint32_t* err) {
    __shared__ uint32_t s_flag[kLocal];
    __shared__ float4 s_lf[2 * kLocal];  // leaf boxes (lo, hi) of the block's leaves
    __shared__ float4 s_in[2 * kLocal];  // boxes of the block's inner nodes
    const uint32_t L0 = blockIdx.x * kLocal;
    const uint32_t L1 = min(L0 + kLocal, n);
    for (uint32_t i = threadIdx.x; i < kLocal; i += kT) s_flag[i] = 0u;
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
        bool local = true;
        while (par != rq::kNoParent) {
            const uint32_t p = par >> 1;
            const int32_t a = kl[p], b = kr[p];
            float4 alo, ahi, blo, bhi;
            if (local && __ldg(klo + p) >= L0 && __ldg(khi + p) < L1) {
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
                // from here up every range crosses a block boundary
                local = false;
                if (rq::atom_add_acq_rel(&refit_flag[p], 1u) == 0u) break;
                const float4* ba = a < 0 ? box_lf + 2 * size_t(uint32_t(a) & 0x7fffffffu) : box_in + 2 * size_t(a);
                const float4* bb = b < 0 ? box_lf + 2 * size_t(uint32_t(b) & 0x7fffffffu) : box_in + 2 * size_t(b);
                alo = rq::ld_cg4(ba);
                ahi = rq::ld_cg4(ba + 1);
                blo = rq::ld_cg4(bb);
                bhi = rq::ld_cg4(bb + 1);
                __stcg(box_in + 2 * size_t(p),
                       make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f));
                __stcg(box_in + 2 * size_t(p) + 1,
                       make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f));
            }
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

size_t rq_build_scratch_carve(void* base, uint32_t n, BuildScratch& s) {
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
    return c.off + 256;
}

int rq_launch_build(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                    uint32_t n, uint32_t max_leaf, bool collapse, cudaStream_t st) {
    BuildScratch s;
    const size_t need = rq_build_scratch_carve(nullptr, n, s);
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    rq_build_scratch_carve(ctx->scratch, n, s);
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
    k_leaves_local<<<(n + kLocal - 1) / kLocal, kT, 0, st>>>(pos, sf, idx, n, max_leaf, skeys, sids, s.kl, s.kr,
                                                             s.klo, s.khi, s.par_in, s.par_lf, s.box_in, s.box_lf,
                                                             s.refit_flag, s.c, bvh->tris, bvh->perm, bvh->skeys,
                                                             ctx->d_err);
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
