// k_median.cu — the reference's median-split build (SoftwareBVH::build,
// common/software_bvh.hpp:35-175) on the GPU, for callers that need its tree
// topology (rq_build with RQ_BUILD_MEDIAN).
//
// The reference recurses: a node over primitives [start, end) is a leaf when
// it holds at most max_leaf of them or when its centroids span less than
// 1e-6 on every axis; otherwise the longest centroid axis (ties keep the
// lower axis) is split at mid = (start + end) / 2 by std::nth_element, the
// left child getting the (mid - start) smallest centroids on that axis.
// Nodes are written depth-first, left child at parent + 1.
//
// Here every level is processed at once.  The primitives are sorted once per
// axis by centroid (stable radix sort of the order-preserving key); a node's
// centroid bounds are then the ends of its three sorted ranges, and its left
// set is the first (mid - start) entries of the range sorted on the chosen
// axis.  A stable partition of all three orders by that membership (one
// scan per axis) keeps every node's ranges sorted for the next level.  When
// no centroid value repeats inside a node on its split axis, the left and
// right sets are the ones nth_element produces, so node boxes, child links,
// leaf offsets and counts equal the reference's; the order inside a leaf
// (left unspecified by nth_element) is the x order.  Sizes and boxes then
// go bottom-up and pre-order positions top-down, level by level.
//
// Everything is stream-ordered (no host synchronisation, so the build can be
// captured in a CUDA graph): splits at mid give children of floor and ceil
// half the count, so the host knows from n and max_leaf alone the deepest
// level a split can reach; it launches every level up to there, and each
// kernel reads the level's frontier size and node range from device memory
// (levels past the tree's real depth find nothing to do).
#include <algorithm>

#include "build_core.cuh"
#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;
constexpr uint32_t kMaxLevels = 96;

struct Seg {
    uint32_t s, e, node;
};

struct MedScratch {
    uint32_t* order[3];
    uint32_t* alt[3];
    uint32_t* flag;     // per primitive: 1 left (or staying), 0 right
    uint32_t* scan;     // exclusive scan of the flags in one axis order
    int32_t* pos_seg;   // per position: frontier index, -1 once in a leaf
    Seg* front[2];
    uint32_t* seg_axis;
    uint32_t* seg_mid;
    uint32_t* seg_split;
    uint32_t* seg_lc;
    uint32_t* seg_rc;
    int32_t* nl;        // left child node id, -1 for a leaf
    int32_t* nr;
    uint32_t* ns;       // primitive range of the node
    uint32_t* ne;
    uint32_t* nsize;    // nodes in the subtree
    uint32_t* npre;     // pre-order position
    float4* nbox;       // 2 per node
    uint32_t* ctl;      // [0] node count
    uint32_t* fcount;   // kMaxLevels + 1: frontier size of each level
    uint32_t* lstart;   // kMaxLevels + 2: first node id of each level
};

size_t carve_med(uintptr_t base, uint32_t n, MedScratch& m) {
    Carve c{base, 0};
    const size_t N = n ? n : 1, M = 2 * N;
    for (int a = 0; a < 3; ++a) m.order[a] = c.take<uint32_t>(N);
    for (int a = 0; a < 3; ++a) m.alt[a] = c.take<uint32_t>(N);
    m.flag = c.take<uint32_t>(N);
    m.scan = c.take<uint32_t>(N);
    m.pos_seg = c.take<int32_t>(N);
    m.front[0] = c.take<Seg>(N);
    m.front[1] = c.take<Seg>(N);
    m.seg_axis = c.take<uint32_t>(N);
    m.seg_mid = c.take<uint32_t>(N);
    m.seg_split = c.take<uint32_t>(N);
    m.seg_lc = c.take<uint32_t>(N);
    m.seg_rc = c.take<uint32_t>(N);
    m.nl = c.take<int32_t>(M);
    m.nr = c.take<int32_t>(M);
    m.ns = c.take<uint32_t>(M);
    m.ne = c.take<uint32_t>(M);
    m.nsize = c.take<uint32_t>(M);
    m.npre = c.take<uint32_t>(M);
    m.nbox = c.take<float4>(2 * M);
    m.ctl = c.take<uint32_t>(8);
    m.fcount = c.take<uint32_t>(kMaxLevels + 1);
    m.lstart = c.take<uint32_t>(kMaxLevels + 2);
    return c.off + 256;
}

inline uint32_t grid(uint32_t n, int sms) {
    const uint32_t b = (n + kT - 1) / kT;
    return std::max(1u, std::min(b, uint32_t(sms) * 8u));
}

__device__ __forceinline__ float comp(const float4& v, uint32_t a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// centroid ((p0+p1)+p2)/3 (software_bvh.hpp:53) and box of every primitive
__global__ void __launch_bounds__(kT) k_med_setup(const float* __restrict__ pos, uint32_t sf,
                                                  const uint32_t* __restrict__ idx, uint32_t n,
                                                  float4* __restrict__ cent, float4* __restrict__ box) {
    for (uint32_t t = blockIdx.x * kT + threadIdx.x; t < n; t += gridDim.x * kT) {
        rq::F3 p0, p1, p2;
        rq::load_tri(pos, sf, idx, t, p0, p1, p2);
        cent[t] = rq::centroid(p0, p1, p2);
        box[2 * t] = make_float4(fminf(fminf(p0.x, p1.x), p2.x), fminf(fminf(p0.y, p1.y), p2.y),
                                 fminf(fminf(p0.z, p1.z), p2.z), 0.0f);
        box[2 * t + 1] = make_float4(fmaxf(fmaxf(p0.x, p1.x), p2.x), fmaxf(fmaxf(p0.y, p1.y), p2.y),
                                     fmaxf(fmaxf(p0.z, p1.z), p2.z), 0.0f);
    }
}

__global__ void __launch_bounds__(kT) k_med_keys(const float4* __restrict__ cent, uint32_t n, uint32_t axis,
                                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint32_t t = blockIdx.x * kT + threadIdx.x; t < n; t += gridDim.x * kT) {
        keys[t] = rq::f2o(comp(cent[t], axis));
        vals[t] = t;
    }
}

__global__ void __launch_bounds__(kT) k_med_init(uint32_t n, MedScratch m) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) m.pos_seg[i] = 0;
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < kMaxLevels + 1; i += gridDim.x * kT) m.fcount[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        m.front[0][0] = Seg{0u, n, 0u};
        m.ns[0] = 0;
        m.ne[0] = n;
        m.ctl[0] = 1;
        m.fcount[0] = 1;
        m.lstart[0] = 0;
        m.lstart[1] = 1;
    }
}

// One frontier node of level L: leaf, or split on the longest centroid axis
// at mid.  The level's frontier size is fcount[L]; children go to level L+1.
__global__ void __launch_bounds__(kT) k_med_decide(const Seg* __restrict__ cur, uint32_t L, uint32_t max_leaf,
                                                   const float4* __restrict__ cent, MedScratch m, Seg* next) {
    const uint32_t j = blockIdx.x * kT + threadIdx.x;
    if (j >= m.fcount[L]) return;
    const Seg g = cur[j];
    m.seg_split[j] = 0;
    const uint32_t cnt = g.e - g.s;
    if (cnt <= max_leaf) {
        m.nl[g.node] = -1;
        return;
    }
    float ext[3];
    for (uint32_t a = 0; a < 3; ++a)
        ext[a] = comp(cent[m.order[a][g.e - 1]], a) - comp(cent[m.order[a][g.s]], a);
    uint32_t axis = 0;
    float mx = ext[0];
    if (ext[1] > mx) {
        axis = 1;
        mx = ext[1];
    }
    if (ext[2] > mx) {
        axis = 2;
        mx = ext[2];
    }
    if (mx < 1e-6f) {
        m.nl[g.node] = -1;
        return;
    }
    const uint32_t mid = (g.s + g.e) / 2;
    const uint32_t id = atomicAdd(m.ctl, 2u);
    m.nl[g.node] = int32_t(id);
    m.nr[g.node] = int32_t(id + 1);
    m.ns[id] = g.s;
    m.ne[id] = mid;
    m.ns[id + 1] = mid;
    m.ne[id + 1] = g.e;
    const uint32_t f = atomicAdd(m.fcount + L + 1, 2u);
    next[f] = Seg{g.s, mid, id};
    next[f + 1] = Seg{mid, g.e, id + 1};
    m.seg_axis[j] = axis;
    m.seg_mid[j] = mid;
    m.seg_lc[j] = f;
    m.seg_rc[j] = f + 1;
    m.seg_split[j] = 1;
}

// Membership of every primitive: left of its node's split (from the order of
// the split axis), or staying (nodes that do not split, finished leaves).
__global__ void __launch_bounds__(kT) k_med_flags(uint32_t n, MedScratch m) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const int32_t j = m.pos_seg[i];
        if (j < 0 || !m.seg_split[j]) {
            m.flag[m.order[0][i]] = 1u;
        } else {
            m.flag[m.order[m.seg_axis[j]][i]] = i < m.seg_mid[j] ? 1u : 0u;
        }
    }
}

// Stable partition of one axis order inside every splitting node.
__global__ void __launch_bounds__(kT) k_med_scatter(uint32_t n, const uint32_t* __restrict__ order,
                                                    uint32_t* __restrict__ out, const Seg* __restrict__ cur,
                                                    MedScratch m) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const uint32_t prim = order[i];
        const int32_t j = m.pos_seg[i];
        if (j < 0 || !m.seg_split[j]) {
            out[i] = prim;
            continue;
        }
        const uint32_t s = cur[j].s, mid = m.seg_mid[j];
        const uint32_t lr = m.scan[i] - m.scan[s];
        out[m.flag[prim] ? s + lr : mid + (i - s - lr)] = prim;
    }
}

// Positions move to their child segment (or leave the frontier); the nodes
// level L's splits created end at the node count, which starts level L+2.
__global__ void __launch_bounds__(kT) k_med_posseg(uint32_t n, uint32_t L, MedScratch m) {
    if (blockIdx.x == 0 && threadIdx.x == 0) m.lstart[L + 2] = m.ctl[0];
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const int32_t j = m.pos_seg[i];
        if (j < 0) continue;
        if (!m.seg_split[j])
            m.pos_seg[i] = -1;
        else
            m.pos_seg[i] = int32_t(i < m.seg_mid[j] ? m.seg_lc[j] : m.seg_rc[j]);
    }
}

// Nodes of level L, [lstart[L], lstart[L+1]): subtree sizes and boxes from
// the level below.
__global__ void __launch_bounds__(kT) k_med_up(uint32_t L, MedScratch m, const float4* __restrict__ pbox,
                                               uint32_t* counts) {
    const uint32_t v = m.lstart[L] + blockIdx.x * kT + threadIdx.x;
    if (v >= m.lstart[L + 1]) return;
    float4 a, b;
    if (m.nl[v] < 0) {
        a = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
        b = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
        for (uint32_t i = m.ns[v]; i < m.ne[v]; ++i) {
            const uint32_t p = m.order[0][i];
            const float4 l = pbox[2 * p], h = pbox[2 * p + 1];
            a = make_float4(fminf(a.x, l.x), fminf(a.y, l.y), fminf(a.z, l.z), 0.0f);
            b = make_float4(fmaxf(b.x, h.x), fmaxf(b.y, h.y), fmaxf(b.z, h.z), 0.0f);
        }
        m.nsize[v] = 1;
        atomicMax(counts + 3, m.ne[v] - m.ns[v]);
    } else {
        const uint32_t l = uint32_t(m.nl[v]), r = uint32_t(m.nr[v]);
        const float4 la = m.nbox[2 * l], lb = m.nbox[2 * l + 1], ra = m.nbox[2 * r], rb = m.nbox[2 * r + 1];
        a = make_float4(fminf(la.x, ra.x), fminf(la.y, ra.y), fminf(la.z, ra.z), 0.0f);
        b = make_float4(fmaxf(lb.x, rb.x), fmaxf(lb.y, rb.y), fmaxf(lb.z, rb.z), 0.0f);
        m.nsize[v] = 1 + m.nsize[l] + m.nsize[r];
    }
    m.nbox[2 * v] = a;
    m.nbox[2 * v + 1] = b;
}

__global__ void __launch_bounds__(kT) k_med_down(uint32_t L, MedScratch m) {
    const uint32_t v = m.lstart[L] + blockIdx.x * kT + threadIdx.x;
    if (v >= m.lstart[L + 1] || m.nl[v] < 0) return;
    const uint32_t l = uint32_t(m.nl[v]), r = uint32_t(m.nr[v]);
    m.npre[l] = m.npre[v] + 1;
    m.npre[r] = m.npre[v] + 1 + m.nsize[l];
}

__global__ void __launch_bounds__(kT) k_med_emit(MedScratch m, rq_bvh2_node* __restrict__ out, uint32_t* counts) {
    const uint32_t nodes = m.ctl[0];
    for (uint32_t v = blockIdx.x * kT + threadIdx.x; v < nodes; v += gridDim.x * kT) {
        const bool leaf = m.nl[v] < 0;
        const int32_t lc = leaf ? int32_t(~m.ns[v]) : int32_t(m.npre[m.nl[v]]);
        const int32_t rc = leaf ? int32_t(m.ne[v] - m.ns[v]) : int32_t(m.npre[m.nr[v]]);
        const float4 a = m.nbox[2 * v], b = m.nbox[2 * v + 1];
        float4* o = reinterpret_cast<float4*>(out + m.npre[v]);
        o[0] = make_float4(a.x, a.y, a.z, __int_as_float(lc));
        o[1] = make_float4(b.x, b.y, b.z, __int_as_float(rc));
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) counts[0] = nodes;
}

__global__ void __launch_bounds__(kT) k_med_tris(const float* __restrict__ pos, uint32_t sf,
                                                 const uint32_t* __restrict__ idx, uint32_t n,
                                                 const uint32_t* __restrict__ order, rq_triangle* __restrict__ tris,
                                                 uint32_t* __restrict__ perm) {
    for (uint32_t i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const uint32_t p = order[i];
        rq::F3 p0, p1, p2;
        rq::load_tri(pos, sf, idx, p, p0, p1, p2);
        float4* t = reinterpret_cast<float4*>(tris + i);
        t[0] = make_float4(p0.x, p0.y, p0.z, 0.0f);
        t[1] = make_float4(p1.x, p1.y, p1.z, 0.0f);
        t[2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
        perm[i] = p;
    }
}

}  // namespace

int rq_launch_build_median(rq_ctx* ctx, rq_bvh* bvh, const float* pos, uint32_t stride_bytes, const uint32_t* idx,
                           uint32_t n, uint32_t max_leaf, bool collapse, cudaStream_t st) {
    BuildScratch s;
    MedScratch m;
    const size_t bs = rq_build_scratch_carve(nullptr, n, s);
    const size_t need = bs + carve_med(0, n, m);
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    rq_build_scratch_carve(ctx->scratch, n, s);
    carve_med(reinterpret_cast<uintptr_t>(ctx->scratch) + ((bs + 255) & ~size_t(255)), n, m);
    const uint32_t sf = stride_bytes / 4;
    const int sms = ctx->num_sms;
    const uint32_t g = grid(n, sms);
    cudaError_t e = cudaMemsetAsync(bvh->d_counts, 0, 4 * sizeof(uint32_t), st);
    k_med_setup<<<g, kT, 0, st>>>(pos, sf, idx, n, s.cent, s.box_lf);
    // one stable sort per axis by centroid
    for (uint32_t a = 0; a < 3 && e == cudaSuccess; ++a) {
        k_med_keys<<<g, kT, 0, st>>>(s.cent, n, a, s.keys[0], s.vals[0]);
        cudaMemsetAsync(s.tile_ctr, 0, 16 * sizeof(uint32_t), st);
        int rb = 0;
        rc = rq_launch_sort(ctx, s, n, 32, st, &rb);
        if (rc) return rc;
        e = cudaMemcpyAsync(m.order[a], s.vals[rb], sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    }
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "median build setup");
    k_med_init<<<g, kT, 0, st>>>(n, m);
    // the deepest level a split can reach: children hold floor and ceil
    // half their parent's count, so the largest count of level L is n halved
    // (rounded up) L times; the level whose largest count fits a leaf is the
    // last one
    uint32_t levels = 1;
    for (uint32_t c = n; c > max_leaf; c = (c + 1) / 2) ++levels;
    if (levels > kMaxLevels) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "median tree deeper than 96 levels");
    // widest possible frontier / level of level L: min(2^L, n) segments
    auto width = [&](uint32_t L) { return L >= 31 ? n : std::min(n, 1u << L); };
    // top-down, one level per round, no host synchronisation
    uint32_t cur = 0;
    for (uint32_t L = 0; L < levels; ++L) {
        k_med_decide<<<(width(L) + kT - 1) / kT, kT, 0, st>>>(m.front[cur], L, max_leaf, s.cent, m,
                                                              m.front[cur ^ 1]);
        k_med_flags<<<g, kT, 0, st>>>(n, m);
        for (int a = 0; a < 3; ++a) {
            // exclusive scan of the membership flags in this axis's order
            cudaMemsetAsync(s.tile_ctr + 8, 0, sizeof(uint32_t), st);
            rq_launch_scan(ctx, m.flag, m.scan, n, s.scan_status, s.tile_ctr + 8, st, m.order[a]);
            k_med_scatter<<<g, kT, 0, st>>>(n, m.order[a], m.alt[a], m.front[cur], m);
            std::swap(m.order[a], m.alt[a]);
        }
        k_med_posseg<<<g, kT, 0, st>>>(n, L, m);
        cur ^= 1u;
    }
    // bottom-up sizes and boxes, top-down pre-order positions (nodes lie on
    // levels 0 .. levels-1, at most min(2^L, n) on level L; a level past the
    // tree's real depth is empty)
    for (uint32_t L = levels; L-- > 0;)
        k_med_up<<<(width(L) + kT - 1) / kT, kT, 0, st>>>(L, m, s.box_lf, bvh->d_counts);
    e = cudaMemsetAsync(m.npre, 0, sizeof(uint32_t), st);
    for (uint32_t L = 0; L < levels && e == cudaSuccess; ++L)
        k_med_down<<<(width(L) + kT - 1) / kT, kT, 0, st>>>(L, m);
    k_med_emit<<<grid(2 * n, sms), kT, 0, st>>>(m, bvh->nodes2, bvh->d_counts);
    k_med_tris<<<g, kT, 0, st>>>(pos, sf, idx, n, m.order[0], bvh->tris, bvh->perm);
    rc = rq_cuda_status(ctx, e == cudaSuccess ? cudaGetLastError() : e, "median build");
    if (rc) return rc;
    if (collapse) return rq_launch_collapse(ctx, bvh, s, st);
    return RQ_OK;
}
