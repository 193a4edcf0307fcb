// k_collapse.cu — binary BVH -> 4-wide BVH with the greedy rule of
// SoftwareBVH4::collapse (common/software_bvh.hpp:202-291): starting from a
// node's two children, repeatedly open the inner candidate with the largest
// surface area 2(dx dy + dy dz + dz dx) (strict >, first wins; the opened
// node's left child takes its slot, its right child is appended) until four
// candidates or none inner.  Output nodes are in the reference's depth-first
// pre-order (a node precedes its subtree; inner children in slot order), so
// the bytes equal fromBVH2's for the same binary BVH.
//
// One persistent cooperative launch, all blocks co-resident:
//   phase 1  top-down, one grid barrier per 4-wide level: candidates of each
//            frontier node, inner candidates appended to a queue;
//   phase 2  bottom-up over the recorded levels: subtree sizes;
//   phase 3  top-down: pre-order index of each child = parent + 1 + sizes of
//            the earlier inner siblings; node and slot-map writes.
// Grid barriers spin with an iteration cap; on timeout they set
// RQ_DERR_GRID_BARRIER and every block leaves the kernel.
#include <algorithm>

#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;
constexpr int kMaxLevels = 120;
constexpr uint32_t kBarrierSpin = 1u << 21;

struct CollapseArgs {
    const rq_bvh2_node* n2;
    uint32_t* counts;
    rq_bvh4_node* out4;
    int32_t* map4;
    uint32_t* q;
    int32_t* cand;
    int32_t* child_q;
    uint32_t* sz;
    uint32_t* pre;
    uint32_t* ctl;  // [0] queue tail [1] barrier arrivals [2] barrier generation
    uint32_t* err;
};

// Returns false if the barrier (or an earlier one, in any block) timed out.
__device__ bool grid_sync(uint32_t* ctl, uint32_t* err) {
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t ok = (rq::ld_relaxed(err) & RQ_DERR_GRID_BARRIER) == 0u;
        if (ok) {
            uint32_t g = rq::ld_acquire(ctl + 2);
            __threadfence();
            uint32_t arrived = atomicAdd(ctl + 1, 1u) + 1u;
            if (arrived == gridDim.x) {
                atomicExch(ctl + 1, 0u);
                __threadfence();
                rq::st_release(ctl + 2, g + 1u);
            } else {
                uint32_t spins = 0;
                while (rq::ld_acquire(ctl + 2) == g) {
                    if (++spins > kBarrierSpin) {
                        rq::set_err(err, RQ_DERR_GRID_BARRIER);
                        ok = 0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0u;
}

struct N2 {
    float mn[3], mx[3];
    int32_t l, r;
};
__device__ __forceinline__ N2 load2(const rq_bvh2_node* n2, int32_t i) {
    const float4* p = reinterpret_cast<const float4*>(n2 + i);
    float4 a = __ldg(p), b = __ldg(p + 1);
    N2 o;
    o.mn[0] = a.x;
    o.mn[1] = a.y;
    o.mn[2] = a.z;
    o.l = __float_as_int(a.w);
    o.mx[0] = b.x;
    o.mx[1] = b.y;
    o.mx[2] = b.z;
    o.r = __float_as_int(b.w);
    return o;
}

__global__ void __launch_bounds__(kT) k_collapse(CollapseArgs A) {
    __shared__ uint32_t s_lvl[kMaxLevels + 2];
    const uint32_t tid = blockIdx.x * kT + threadIdx.x;
    const uint32_t nthreads = gridDim.x * kT;
    const bool root_leaf = load2(A.n2, 0).l < 0;
    if (tid == 0) {
        A.q[0] = 0u;
        A.pre[0] = 0u;
        A.ctl[0] = 1u;
    }
    if (!grid_sync(A.ctl, A.err)) return;

    // ---- phase 1: levels, candidates, queue
    uint32_t start = 0, end = 1, depth = 0;
    while (start < end) {
        if (threadIdx.x == 0) s_lvl[depth] = start;
        for (uint32_t e = start + tid; e < end; e += nthreads) {
            int32_t u = int32_t(__ldcg(A.q + e));
            int32_t c[4] = {-1, -1, -1, -1};
            int nc;
            if (root_leaf) {
                c[0] = 0;
                nc = 1;
            } else {
                N2 nd = load2(A.n2, u);
                c[0] = nd.l;
                c[1] = nd.r;
                nc = 2;
                while (nc < 4) {
                    int best = -1;
                    float best_sa = -1.0f;
                    for (int i = 0; i < nc; ++i) {
                        N2 ci = load2(A.n2, c[i]);
                        if (ci.l >= 0) {
                            float dx = ci.mx[0] - ci.mn[0];
                            float dy = ci.mx[1] - ci.mn[1];
                            float dz = ci.mx[2] - ci.mn[2];
                            float sa = 2.0f * ((dx * dy + dy * dz) + dz * dx);
                            if (sa > best_sa) {
                                best_sa = sa;
                                best = i;
                            }
                        }
                    }
                    if (best < 0) break;
                    N2 ex = load2(A.n2, c[best]);
                    c[best] = ex.l;
                    c[nc++] = ex.r;
                }
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int32_t cq = -1;
                if (c[k] >= 0 && !root_leaf && load2(A.n2, c[k]).l >= 0) {
                    uint32_t pos = atomicAdd(A.ctl, 1u);
                    __stcg(A.q + pos, uint32_t(c[k]));
                    cq = int32_t(pos);
                }
                __stcg(A.cand + 4 * size_t(e) + k, c[k]);
                __stcg(A.child_q + 4 * size_t(e) + k, cq);
            }
        }
        if (!grid_sync(A.ctl, A.err)) return;
        ++depth;
        start = end;
        end = __ldcg(A.ctl);
        if (depth >= kMaxLevels) {
            if (tid == 0) rq::set_err(A.err, RQ_DERR_QUEUE);
            return;
        }
    }
    if (threadIdx.x == 0) s_lvl[depth] = end;
    __syncthreads();
    const uint32_t total = end;

    // ---- phase 2: subtree sizes, deepest level first
    for (int lv = int(depth) - 1; lv >= 0; --lv) {
        for (uint32_t e = s_lvl[lv] + tid; e < s_lvl[lv + 1]; e += nthreads) {
            uint32_t s = 1;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int32_t cq = __ldcg(A.child_q + 4 * size_t(e) + k);
                if (cq >= 0) s += __ldcg(A.sz + cq);
            }
            __stcg(A.sz + e, s);
        }
        if (!grid_sync(A.ctl, A.err)) return;
    }

    // ---- phase 3: pre-order positions and node writes, top-down
    for (uint32_t lv = 0; lv < depth; ++lv) {
        for (uint32_t e = s_lvl[lv] + tid; e < s_lvl[lv + 1]; e += nthreads) {
            uint32_t p = __ldcg(A.pre + e);
            uint32_t off = p + 1u;
            float mnx[4], mxx[4], mny[4], mxy[4], mnz[4], mxz[4];
            int32_t ci[4], cc[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                int32_t c = __ldcg(A.cand + 4 * size_t(e) + k);
                mnx[k] = mxx[k] = mny[k] = mxy[k] = mnz[k] = mxz[k] = 0.0f;
                ci[k] = 0;
                cc[k] = 0;
                if (c >= 0) {
                    N2 nd = load2(A.n2, c);
                    mnx[k] = nd.mn[0];
                    mxx[k] = nd.mx[0];
                    mny[k] = nd.mn[1];
                    mxy[k] = nd.mx[1];
                    mnz[k] = nd.mn[2];
                    mxz[k] = nd.mx[2];
                    int32_t cq = __ldcg(A.child_q + 4 * size_t(e) + k);
                    if (cq >= 0) {
                        __stcg(A.pre + cq, off);
                        ci[k] = int32_t(off);
                        cc[k] = -1;
                        off += __ldcg(A.sz + cq);
                    } else {
                        ci[k] = nd.l;
                        cc[k] = nd.r;
                    }
                }
                A.map4[4 * size_t(p) + k] = c;
            }
            float4* o = reinterpret_cast<float4*>(A.out4 + p);
            o[0] = make_float4(mnx[0], mnx[1], mnx[2], mnx[3]);
            o[1] = make_float4(mxx[0], mxx[1], mxx[2], mxx[3]);
            o[2] = make_float4(mny[0], mny[1], mny[2], mny[3]);
            o[3] = make_float4(mxy[0], mxy[1], mxy[2], mxy[3]);
            o[4] = make_float4(mnz[0], mnz[1], mnz[2], mnz[3]);
            o[5] = make_float4(mxz[0], mxz[1], mxz[2], mxz[3]);
            reinterpret_cast<int4*>(o)[6] = make_int4(ci[0], ci[1], ci[2], ci[3]);
            reinterpret_cast<int4*>(o)[7] = make_int4(cc[0], cc[1], cc[2], cc[3]);
        }
        if (!grid_sync(A.ctl, A.err)) return;
    }
    if (tid == 0) {
        A.counts[1] = total;
        A.counts[2] = depth;
    }
}

}  // namespace

int rq_collapse_blocks(int device, int num_sms) {
    int per_sm = 0;
    cudaSetDevice(device);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_collapse, kT, 0) != cudaSuccess) return 0;
    if (per_sm > 2) per_sm = 2;
    return per_sm * num_sms;
}

int rq_launch_collapse(rq_ctx* ctx, rq_bvh* bvh, BuildScratch& s, cudaStream_t st) {
    if (ctx->collapse_blocks <= 0) return rq_set_error(ctx, RQ_ERR_CUDA, "collapse kernel cannot be co-resident");
    cudaMemsetAsync(s.coll_ctl, 0, 256 * sizeof(uint32_t), st);
    CollapseArgs a;
    a.n2 = bvh->nodes2;
    a.counts = bvh->d_counts;
    a.out4 = bvh->nodes4;
    a.map4 = bvh->map4;
    a.q = s.q;
    a.cand = s.cand;
    a.child_q = s.child_q;
    a.sz = s.sz;
    a.pre = s.pre;
    a.ctl = s.coll_ctl;
    a.err = ctx->d_err;
    void* args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((void*)k_collapse, dim3(ctx->collapse_blocks), dim3(kT), args, 0, st);
    return rq_cuda_status(ctx, e, "collapse launch");
}

// ------------------------------------------------------------------------
// Checks of imported trees: largest leaf, 4-wide depth, index ranges.  A
// malformed tree sets counts[3] to 0xFFFFFFFF, which the importers reject.
namespace {

constexpr uint32_t kNoParent = 0xffffffffu;

__global__ void __launch_bounds__(kT) k_analyze2(const rq_bvh2_node* __restrict__ n2, uint32_t* counts,
                                                 uint32_t ntri) {
    const uint32_t m = counts[0];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < m; i += gridDim.x * kT) {
        const rq_bvh2_node nd = n2[i];
        bool bad;
        if (nd.left_child < 0) {
            uint32_t first = uint32_t(~nd.left_child);
            bad = nd.right_child <= 0 || uint64_t(first) + uint64_t(nd.right_child) > ntri;
            if (!bad) atomicMax(&counts[3], uint32_t(nd.right_child));
        } else {
            bad = uint32_t(nd.left_child) >= m || nd.right_child < 0 || uint32_t(nd.right_child) >= m;
        }
        if (bad) atomicExch(&counts[3], 0xffffffffu);
    }
}

__global__ void __launch_bounds__(kT) k_parent4(const rq_bvh4_node* __restrict__ n4, const uint32_t* counts,
                                                uint32_t* __restrict__ parent) {
    const uint32_t m = counts[1];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < m; i += gridDim.x * kT) {
        if (i == 0) parent[0] = kNoParent;
        for (int k = 0; k < 4; ++k)
            if (n4[i].child_count[k] < 0) {
                uint32_t c = uint32_t(n4[i].child_index[k]);
                if (c < m && c != 0) parent[c] = i;
            }
    }
}

__global__ void __launch_bounds__(kT) k_depth4(const rq_bvh4_node* __restrict__ n4, const uint32_t* __restrict__ parent,
                                               uint32_t* counts, uint32_t ntri) {
    const uint32_t m = counts[1];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < m; i += gridDim.x * kT) {
        bool bad = false;
        for (int k = 0; k < 4; ++k) {
            int32_t cc = n4[i].child_count[k], ci = n4[i].child_index[k];
            if (cc < 0) {
                bad |= cc != -1 || ci <= 0 || uint32_t(ci) >= m;
            } else if (cc > 0) {
                uint32_t first = uint32_t(~ci);
                bad |= uint64_t(first) + uint64_t(cc) > ntri;
                if (!bad) atomicMax(&counts[3], uint32_t(cc));
            }
        }
        uint32_t d = 1, p = i == 0 ? kNoParent : parent[i];
        while (p != kNoParent && d <= m) {
            ++d;
            p = p == 0 ? kNoParent : parent[p];
        }
        if (d > m) bad = true;
        atomicMax(&counts[2], d);
        if (bad) atomicExch(&counts[3], 0xffffffffu);
    }
}

}  // namespace

int rq_launch_analyze2(rq_ctx* ctx, rq_bvh* bvh, cudaStream_t st) {
    uint32_t blocks = std::min<uint32_t>((bvh->cap_nodes2 + kT - 1) / kT, uint32_t(ctx->num_sms) * 8u);
    k_analyze2<<<blocks ? blocks : 1, kT, 0, st>>>(bvh->nodes2, bvh->d_counts, bvh->num_tris);
    return rq_cuda_status(ctx, cudaGetLastError(), "bvh2 analysis launch");
}

int rq_launch_analyze4(rq_ctx* ctx, rq_bvh* bvh, cudaStream_t st) {
    int rc = rq_ensure_scratch(ctx, sizeof(uint32_t) * (size_t(bvh->cap_nodes4) + 64), st);
    if (rc) return rc;
    uint32_t* parent = static_cast<uint32_t*>(ctx->scratch);
    // parents of unreachable nodes stay unset: mark everything "no parent"
    cudaMemsetAsync(parent, 0xff, sizeof(uint32_t) * bvh->cap_nodes4, st);
    uint32_t blocks = std::min<uint32_t>((bvh->cap_nodes4 + kT - 1) / kT, uint32_t(ctx->num_sms) * 8u);
    if (!blocks) blocks = 1;
    k_parent4<<<blocks, kT, 0, st>>>(bvh->nodes4, bvh->d_counts, parent);
    k_depth4<<<blocks, kT, 0, st>>>(bvh->nodes4, parent, bvh->d_counts, bvh->num_tris);
    return rq_cuda_status(ctx, cudaGetLastError(), "bvh4 analysis launch");
}
