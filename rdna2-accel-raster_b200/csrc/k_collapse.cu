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
//   phase 1  top-down, one grid barrier per 4-wide level (the narrow top
//            levels by one block): candidates of each frontier node, inner
//            candidates appended to a queue;
//   phase 2  subtree sizes bottom-up by atomic arrival counts (no barrier per
//            level);
//   phase 3  each node's pre-order index from its ancestors' sibling sizes
//            (no barrier per level); node and slot-map writes.
// Grid barriers spin with an iteration cap; on timeout they set
// RQ_DERR_GRID_BARRIER and every block leaves the kernel.
#include <algorithm>

#include "build_core.cuh"
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
    uint32_t* par;
    unsigned long long* acc;
    uint32_t* ctl;  // [1] barrier arrivals [2] barrier generation, [4..10] collapse_levels control
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
                ok = rq::wait_change(ctl + 2, g, kBarrierSpin, err, RQ_DERR_GRID_BARRIER) ? 1u : 0u;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0u;
}

__global__ void __launch_bounds__(kT) k_collapse(CollapseArgs A) {
    __shared__ uint32_t s_lvl[kMaxLevels + 2];
    rq::CollapseIO io;
    io.n2 = A.n2;
    io.q = A.q;
    io.cand = A.cand;
    io.child_q = A.child_q;
    io.sz = A.sz;
    io.par = A.par;
    io.acc = A.acc;
    io.tail = A.ctl;
    io.out4 = A.out4;
    io.map4 = A.map4;
    uint32_t total = 0, depth = 0;
    auto sync = [&]() { return grid_sync(A.ctl, A.err); };
    // levels of at most 256 entries by block 0 alone (measured: a little faster than a grid barrier each)
    if (!rq::collapse_levels<true, false, 256>(io, blockIdx.x * kT + threadIdx.x, gridDim.x * kT, s_lvl, kMaxLevels,
                                               sync, A.err, &total, &depth))
        return;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
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
    a.par = s.cpar;
    a.acc = s.cacc;
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
