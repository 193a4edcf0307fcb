// build_core.cuh — the per-element steps of the LBVH build, shared by the
// grid-wide kernels of k_build.cu / k_collapse.cu (one mesh per launch) and
// the block-level pipeline of k_batch.cu (one mesh per thread block, many
// meshes per launch).  Both call these functions, so a mesh built either way
// has the same bytes.
//
// Loads of data written earlier in the same launch use plain (coherent)
// loads; only the caller's vertex and index buffers go through __ldg.
#pragma once

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

constexpr uint32_t kNoParent = 0xffffffffu;

__device__ __forceinline__ void load_tri(const float* __restrict__ pos, uint32_t sf, const uint32_t* __restrict__ idx,
                                         uint32_t t, F3& p0, F3& p1, F3& p2) {
    uint32_t i0, i1, i2;
    if (idx) {
        i0 = __ldg(idx + 3ull * t);
        i1 = __ldg(idx + 3ull * t + 1);
        i2 = __ldg(idx + 3ull * t + 2);
    } else {
        i0 = 3 * t;
        i1 = 3 * t + 1;
        i2 = 3 * t + 2;
    }
    const float* a = pos + size_t(i0) * sf;
    const float* b = pos + size_t(i1) * sf;
    const float* c = pos + size_t(i2) * sf;
    p0 = {__ldg(a), __ldg(a + 1), __ldg(a + 2)};
    p1 = {__ldg(b), __ldg(b + 1), __ldg(b + 2)};
    p2 = {__ldg(c), __ldg(c + 1), __ldg(c + 2)};
}

// Centroid exactly as SoftwareBVH::build (common/software_bvh.hpp:53).
__device__ __forceinline__ float4 centroid(F3 p0, F3 p1, F3 p2) {
    return make_float4(((p0.x + p1.x) + p2.x) / 3.0f, ((p0.y + p1.y) + p2.y) / 3.0f, ((p0.z + p1.z) + p2.z) / 3.0f,
                       0.0f);
}

// Scale of the Morton grid: 1024 cells over the largest centroid extent.
__device__ __forceinline__ float morton_scale(float lx, float ly, float lz, float hx, float hy, float hz) {
    const float ext = fmaxf(fmaxf(hx - lx, hy - ly), hz - lz);
    return ext > 1e-30f ? 1024.0f / ext : 0.0f;
}

__device__ __forceinline__ uint32_t morton30(float4 c, float lx, float ly, float lz, float scale) {
    return expand10(quantize10(c.x, lx, scale)) * 4u + expand10(quantize10(c.y, ly, scale)) * 2u +
           expand10(quantize10(c.z, lz, scale));
}

__device__ __forceinline__ int kdelta(const uint32_t* k, int n, int i, int j) {
    if (j < 0 || j > n - 1) return -1;
    const uint32_t x = k[i] ^ k[j];
    if (x) return __clz(x);
    return 32 + __clz(uint32_t(i) ^ uint32_t(j));
}

// Karras 2012, internal node i of n sorted keys: children (bit 31 = leaf),
// range, and the parent links of both children ((parent << 1) | is_right).
__device__ __forceinline__ void karras_node(const uint32_t* keys, int n, int i, int32_t* kl, int32_t* kr,
                                            uint32_t* klo, uint32_t* khi, uint32_t* par_in, uint32_t* par_lf) {
    const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = kdelta(keys, n, i, i - d);
    int lmax = 2;
    while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = kdelta(keys, n, i, j);
    int s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    const int gamma = i + s * d + min(d, 0);
    const int lo = min(i, j), hi = max(i, j);
    const bool lleaf = lo == gamma, rleaf = hi == gamma + 1;
    kl[i] = lleaf ? int32_t(0x80000000u | uint32_t(gamma)) : gamma;
    kr[i] = rleaf ? int32_t(0x80000000u | uint32_t(gamma + 1)) : gamma + 1;
    klo[i] = uint32_t(lo);
    khi[i] = uint32_t(hi);
    const uint32_t pl = uint32_t(i) << 1, pr = (uint32_t(i) << 1) | 1u;
    if (lleaf)
        par_lf[gamma] = pl;
    else
        par_in[gamma] = pl;
    if (rleaf)
        par_lf[gamma + 1] = pr;
    else
        par_in[gamma + 1] = pr;
    if (i == 0) par_in[0] = kNoParent;
}

__device__ __forceinline__ uint32_t count_in(const uint32_t* klo, const uint32_t* khi, uint32_t i) {
    return khi[i] - klo[i] + 1u;
}

// Sorted leaf k: leaf-ordered triangle copy, permutation, sorted key, leaf box,
// and the depth-first emission count of the leaf starting at k: the emitted
// leaf holding k is its highest ancestor with count <= max_leaf; if it starts
// at k, c = 1 + (consecutive left-child links above it).
__device__ __forceinline__ void leaf_step(uint32_t k, const float* __restrict__ pos, uint32_t sf,
                                          const uint32_t* __restrict__ idx, uint32_t max_leaf, const uint32_t* skeys,
                                          const uint32_t* sids, const uint32_t* klo, const uint32_t* khi,
                                          const uint32_t* par_in, const uint32_t* par_lf, float4* box_lf,
                                          uint32_t* c_out, rq_triangle* tris, uint32_t* perm, uint32_t* keys_out) {
    const uint32_t id = sids[k];
    F3 p0, p1, p2;
    load_tri(pos, sf, idx, id, p0, p1, p2);
    float4* tp = reinterpret_cast<float4*>(tris + k);
    tp[0] = make_float4(p0.x, p0.y, p0.z, 0.0f);
    tp[1] = make_float4(p1.x, p1.y, p1.z, 0.0f);
    tp[2] = make_float4(p2.x, p2.y, p2.z, 0.0f);
    perm[k] = id;
    keys_out[k] = skeys[k];
    box_lf[2 * size_t(k)] = make_float4(fminf(p0.x, fminf(p1.x, p2.x)), fminf(p0.y, fminf(p1.y, p2.y)),
                                        fminf(p0.z, fminf(p1.z, p2.z)), 0.0f);
    box_lf[2 * size_t(k) + 1] = make_float4(fmaxf(p0.x, fmaxf(p1.x, p2.x)), fmaxf(p0.y, fmaxf(p1.y, p2.y)),
                                            fmaxf(p0.z, fmaxf(p1.z, p2.z)), 0.0f);
    uint32_t par = par_lf[k];
    uint32_t ulo = k;
    while (par != kNoParent) {
        const uint32_t pp = par >> 1;
        if (count_in(klo, khi, pp) > max_leaf) break;
        ulo = klo[pp];
        par = par_in[pp];
    }
    uint32_t c = 0;
    if (ulo == k) {
        uint32_t L = 0;
        while (par != kNoParent && (par & 1u) == 0u) {
            ++L;
            par = par_in[par >> 1];
        }
        c = 1u + L;
    }
    c_out[k] = c;
}

// Atomic bottom-up refit from sorted leaf k: at each node the second child
// to arrive computes the union box and continues upward.  The arrival count
// is an acquire-release add: it publishes the box this thread wrote last
// (the leaf box, then each union) and, for the second arrival, makes the
// sibling's box visible.  CTA: all leaves of the tree are in this block.
template <bool CTA = false>
__device__ __forceinline__ void refit_walk(uint32_t k, const int32_t* kl, const int32_t* kr, const uint32_t* par_in,
                                           const uint32_t* par_lf, float4* box_in, const float4* box_lf,
                                           uint32_t* refit_flag, uint32_t* err) {
    uint32_t par = par_lf[k];
    uint32_t guard = 0;
    while (par != kNoParent) {
        const uint32_t p = par >> 1;
        if (atom_add_acq_rel<CTA>(&refit_flag[p], 1u) == 0u) break;
        const int32_t a = kl[p], b = kr[p];
        const float4* ba = a < 0 ? box_lf + 2 * size_t(uint32_t(a) & 0x7fffffffu) : box_in + 2 * size_t(a);
        const float4* bb = b < 0 ? box_lf + 2 * size_t(uint32_t(b) & 0x7fffffffu) : box_in + 2 * size_t(b);
        const float4 alo = ld_cg4(ba), ahi = ld_cg4(ba + 1);
        const float4 blo = ld_cg4(bb), bhi = ld_cg4(bb + 1);
        __stcg(box_in + 2 * size_t(p), make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f));
        __stcg(box_in + 2 * size_t(p) + 1,
               make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f));
        par = par_in[p];
        if (++guard > 128u) {
            set_err(err, RQ_DERR_REFIT);
            break;
        }
    }
}

// Depth-first pre-order node writes for primitive position p: internal node
// p (if emitted) sits at A[lo] + L, the emitted leaf starting at p (if any)
// at A[p] + c[p] - 1.  Returns c[p].
__device__ __forceinline__ uint32_t emit_step(uint32_t p, uint32_t n, uint32_t max_leaf, const int32_t* kr,
                                              const uint32_t* klo, const uint32_t* khi, const uint32_t* par_in,
                                              const uint32_t* par_lf, const float4* box_in, const float4* box_lf,
                                              const uint32_t* c, const uint32_t* A, rq_bvh2_node* out) {
    if (p + 1 < n && count_in(klo, khi, p) > max_leaf) {
        uint32_t L = 0, par = par_in[p];
        while (par != kNoParent && (par & 1u) == 0u) {
            ++L;
            par = par_in[par >> 1];
        }
        const uint32_t pre = A[klo[p]] + L;
        const int32_t r = kr[p];
        const uint32_t rlo = r < 0 ? (uint32_t(r) & 0x7fffffffu) : klo[r];
        // refit boxes were stored with st.cg: read them from L2
        const float4 lo = ld_cg4(box_in + 2 * size_t(p)), hi = ld_cg4(box_in + 2 * size_t(p) + 1);
        float4* o = reinterpret_cast<float4*>(out + pre);
        o[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(int32_t(pre + 1)));
        o[1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(int32_t(A[rlo])));
    }
    const uint32_t cp = c[p];
    if (cp) {
        uint32_t par = par_lf[p];
        uint32_t node = p;
        bool is_leaf = true;
        while (par != kNoParent) {
            const uint32_t pp = par >> 1;
            if (count_in(klo, khi, pp) > max_leaf) break;
            node = pp;
            is_leaf = false;
            par = par_in[pp];
        }
        const uint32_t cnt = is_leaf ? 1u : count_in(klo, khi, node);
        const float4* b = is_leaf ? box_lf + 2 * size_t(node) : box_in + 2 * size_t(node);
        const float4 lo = ld_cg4(b), hi = ld_cg4(b + 1);
        const uint32_t pre = A[p] + cp - 1u;
        float4* o = reinterpret_cast<float4*>(out + pre);
        o[0] = make_float4(lo.x, lo.y, lo.z, __int_as_float(~int32_t(p)));
        o[1] = make_float4(hi.x, hi.y, hi.z, __int_as_float(int32_t(cnt)));
    }
    return cp;
}

// ------------------------------------------------------------- collapse
struct N2 {
    float mn[3], mx[3];
    int32_t l, r;
};

template <bool NC>
__device__ __forceinline__ N2 load_n2(const rq_bvh2_node* n2, int32_t i) {
    const float4* p = reinterpret_cast<const float4*>(n2 + i);
    const float4 a = NC ? __ldg(p) : p[0], b = NC ? __ldg(p + 1) : p[1];
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

// Greedy candidates of SoftwareBVH4::collapse (software_bvh.hpp:225-247)
// for inner binary node u: open the inner candidate with the largest
// surface area (strict >, first wins) until four.  Returns the count;
// inner[i]: candidate i is an inner binary node.
template <bool NC>
__device__ __forceinline__ int greedy_candidates(const rq_bvh2_node* n2, int32_t u, int32_t c[4], bool inner[4]) {
    // each candidate's children and surface area, loaded once (slots are
    // static indices, so the records stay in registers)
    int32_t cl[4], cr[4];
    float sa[4];
    auto set = [&](int i, int32_t id, const N2& nd) {
        c[i] = id;
        cl[i] = nd.l;
        cr[i] = nd.r;
        const float dx = nd.mx[0] - nd.mn[0];
        const float dy = nd.mx[1] - nd.mn[1];
        const float dz = nd.mx[2] - nd.mn[2];
        sa[i] = 2.0f * ((dx * dy + dy * dz) + dz * dx);
    };
    const N2 nd = load_n2<NC>(n2, u);
    {
        const N2 a = load_n2<NC>(n2, nd.l), b = load_n2<NC>(n2, nd.r);
        set(0, nd.l, a);
        set(1, nd.r, b);
    }
    c[2] = c[3] = -1;
    cl[2] = cl[3] = -1;
    cr[2] = cr[3] = -1;
    sa[2] = sa[3] = 0.0f;
    int nc = 2;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        int best = -1;
        float best_sa = -1.0f;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i < nc && cl[i] >= 0 && sa[i] > best_sa) {
                best_sa = sa[i];
                best = i;
            }
        if (best < 0) break;
        int32_t l = 0, r = 0;
#pragma unroll
        for (int i = 0; i < 4; ++i)
            if (i == best) {
                l = cl[i];
                r = cr[i];
            }
        const N2 a = load_n2<NC>(n2, l), b = load_n2<NC>(n2, r);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (i == best) set(i, l, a);
            if (i == nc) set(i, r, b);
        }
        ++nc;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) inner[i] = i < nc && cl[i] >= 0;
    return nc;
}

// Writes 4-wide node p from its candidates; inner children get pre-order
// positions p+1, p+1 + size(first inner child), ... (sizes by queue index).
template <bool NC, class SizeOf, class PreOut>
__device__ __forceinline__ void write_node4(const rq_bvh2_node* n2, const int32_t cand[4], const int32_t cq[4],
                                            uint32_t p, SizeOf size_of, PreOut pre_out, rq_bvh4_node* out4,
                                            int32_t* map4) {
    uint32_t off = p + 1u;
    float mnx[4], mxx[4], mny[4], mxy[4], mnz[4], mxz[4];
    int32_t ci[4], cc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        mnx[k] = mxx[k] = mny[k] = mxy[k] = mnz[k] = mxz[k] = 0.0f;
        ci[k] = 0;
        cc[k] = 0;
        if (cand[k] >= 0) {
            const N2 nd = load_n2<NC>(n2, cand[k]);
            mnx[k] = nd.mn[0];
            mxx[k] = nd.mx[0];
            mny[k] = nd.mn[1];
            mxy[k] = nd.mx[1];
            mnz[k] = nd.mn[2];
            mxz[k] = nd.mx[2];
            if (cq[k] >= 0) {
                pre_out(cq[k], off);
                ci[k] = int32_t(off);
                cc[k] = -1;
                off += size_of(cq[k]);
            } else {
                ci[k] = nd.l;
                cc[k] = nd.r;
            }
        }
        map4[4 * size_t(p) + k] = cand[k];
    }
    float4* o = reinterpret_cast<float4*>(out4 + p);
    o[0] = make_float4(mnx[0], mnx[1], mnx[2], mnx[3]);
    o[1] = make_float4(mxx[0], mxx[1], mxx[2], mxx[3]);
    o[2] = make_float4(mny[0], mny[1], mny[2], mny[3]);
    o[3] = make_float4(mxy[0], mxy[1], mxy[2], mxy[3]);
    o[4] = make_float4(mnz[0], mnz[1], mnz[2], mnz[3]);
    o[5] = make_float4(mxz[0], mxz[1], mxz[2], mxz[3]);
    reinterpret_cast<int4*>(o)[6] = make_int4(ci[0], ci[1], ci[2], ci[3]);
    reinterpret_cast<int4*>(o)[7] = make_int4(cc[0], cc[1], cc[2], cc[3]);
}

// Scratch and outputs of one collapse.
struct CollapseIO {
    const rq_bvh2_node* n2;
    uint32_t* q;        // queue: binary node of each 4-wide node, level by level
    int32_t* cand;      // 4 per queue entry
    int32_t* child_q;   // 4 per queue entry: queue index of inner children, -1
    uint32_t* sz;       // subtree sizes
    uint32_t* par;      // per queue entry: (parent entry << 2) | slot, kNoParent for the root
    unsigned long long* acc;  // per queue entry: (arrived inner children << 32) | their summed sizes
    uint32_t* tail;     // control words: [4..6] per-level append counts, [8..10] hand-over
    rq_bvh4_node* out4;
    int32_t* map4;
};

// Inner children (queue entries) of entry e.
__device__ __forceinline__ uint32_t inner_children(const CollapseIO& io, uint32_t e) {
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) c += __ldcg(io.child_q + 4 * size_t(e) + k) >= 0 ? 1u : 0u;
    return c;
}

// The three phases of the collapse, run by `nthreads` cooperating threads
// (index tid) that meet at `sync()` (false = a barrier gave up; abort):
//   1. top-down per level: candidates, inner candidates appended to q with
//      their parent link;
//   2. subtree sizes bottom-up without level barriers: each entry with no
//      inner children starts a walk; at each parent one 64-bit atomic adds
//      (one arrival, the child's size) and returns the earlier arrivals and
//      sizes, so the arrival that completes the parent carries its size on;
//   3. every entry's pre-order position is the sum over its ancestors of
//      1 + the sizes of the earlier inner siblings (a walk up that stops at
//      the first ancestor whose position a written parent already
//      published), then the node write.
// LEVELS: phases 2 and 3 level by level instead (bottom-up sizes, then
// top-down positions, one sync per level; `acc` holds the positions) — the
// faster form when sync() is a block barrier.  NARROW > 0 (grid-wide use):
// block 0 alone expands the top levels while they hold at most NARROW
// entries.  io.tail holds 16 control words.
// s_lvl (shared, max_levels + 2 entries) records the level boundaries.
// Data written inside the collapse is read with ld.cg: other blocks wrote it.
template <bool NC, bool LEVELS, uint32_t NARROW, class Sync>
__device__ __forceinline__ bool collapse_levels(const CollapseIO& io, uint32_t tid, uint32_t nthreads,
                                                uint32_t* s_lvl, uint32_t max_levels, Sync sync, uint32_t* err,
                                                uint32_t* total_out, uint32_t* depth_out) {
    const bool root_leaf = load_n2<NC>(io.n2, 0).l < 0;
    // Entries of level L+1 are appended at end(L) + an atomic count of their
    // own, io.tail[4 + L % 3]: after the level's sync every thread reads that
    // count while the next level appends to another one, and the one after
    // that is cleared during level L, two syncs after its last reader.
    uint32_t* lvl_cnt = io.tail + 4;
    // Inner candidates take consecutive queue entries: one atomic per warp
    // (the lanes that expand together), each lane's entries after the lower
    // lanes'.  Entry numbers only name queue records; the output does not
    // depend on them.
    auto expand = [&](uint32_t e, uint32_t end, uint32_t depth) {
        const int32_t u = int32_t(__ldcg(io.q + e));
        int32_t c[4] = {-1, -1, -1, -1};
        bool inner[4] = {false, false, false, false};
        if (root_leaf)
            c[0] = 0;
        else
            greedy_candidates<NC>(io.n2, u, c, inner);
        const uint32_t cnt = uint32_t(inner[0]) + uint32_t(inner[1]) + uint32_t(inner[2]) + uint32_t(inner[3]);
        const uint32_t act = __activemask();
        const uint32_t lane = threadIdx.x & 31u, lt = (1u << lane) - 1u;
        const uint32_t b0 = __ballot_sync(act, cnt & 1u), b1 = __ballot_sync(act, cnt & 2u),
                       b2 = __ballot_sync(act, cnt & 4u);
        const uint32_t below = __popc(b0 & lt) + 2u * __popc(b1 & lt) + 4u * __popc(b2 & lt);
        const uint32_t total = __popc(b0) + 2u * __popc(b1) + 4u * __popc(b2);
        const uint32_t leader = __ffs(act) - 1u;
        uint32_t base = 0;
        if (lane == leader && total) base = atomicAdd(lvl_cnt + depth % 3u, total);
        uint32_t pos = end + __shfl_sync(act, base, leader) + below;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            int32_t cq = -1;
            if (inner[k]) {
                __stcg(io.q + pos, uint32_t(c[k]));
                __stcg(io.par + pos, (e << 2) | uint32_t(k));
                __stcg(io.acc + pos, 0ull);
                cq = int32_t(pos++);
            }
            __stcg(io.cand + 4 * size_t(e) + k, c[k]);
            __stcg(io.child_q + 4 * size_t(e) + k, cq);
        }
    };
    if (tid == 0) {
        __stcg(io.q, 0u);
        __stcg(io.par, kNoParent);
        __stcg(io.acc, 0ull);
        atomicExch(lvl_cnt, 0u);
    }
    if (!sync()) return false;
    uint32_t start = 0, end = 1, depth = 0;
    if (NARROW > 0) {
        // the narrow top levels (at most NARROW entries each) by block 0
        // alone, with block barriers; then one sync hands the frontier over
        if (blockIdx.x == 0) {
            while (start < end && end - start <= NARROW && depth + 1 < max_levels) {
                if (threadIdx.x == 0) atomicExch(lvl_cnt + (depth + 1) % 3u, 0u);
                for (uint32_t e = start + threadIdx.x; e < end; e += blockDim.x) expand(e, end, depth);
                __syncthreads();
                const uint32_t n = __ldcg(lvl_cnt + depth % 3u);
                ++depth;
                start = end;
                end += n;
            }
            if (threadIdx.x == 0) {
                __stcg(io.tail + 8, start);
                __stcg(io.tail + 9, end);
                __stcg(io.tail + 10, depth);
            }
        }
        if (!sync()) return false;
        start = __ldcg(io.tail + 8);
        end = __ldcg(io.tail + 9);
        depth = __ldcg(io.tail + 10);
    }
    while (start < end) {
        if (threadIdx.x == 0) s_lvl[depth] = start;
        if (tid == 0) atomicExch(lvl_cnt + (depth + 1) % 3u, 0u);
        for (uint32_t e = start + tid; e < end; e += nthreads) expand(e, end, depth);
        if (!sync()) return false;
        const uint32_t n = __ldcg(lvl_cnt + depth % 3u);
        ++depth;
        start = end;
        end += n;
        if (depth >= max_levels) {
            if (tid == 0) set_err(err, RQ_DERR_QUEUE);
            return false;
        }
    }
    if (threadIdx.x == 0) s_lvl[depth] = end;
    struct SizeOf {
        const uint32_t* sz;
        __device__ uint32_t operator()(int32_t i) const { return __ldcg(sz + i); }
    };
    if constexpr (LEVELS) {
        __syncthreads();
        uint32_t* pre = reinterpret_cast<uint32_t*>(io.acc);  // acc[0] = 0: the root at 0
        for (int lv = int(depth) - 1; lv >= 0; --lv) {
            for (uint32_t e = s_lvl[lv] + tid; e < s_lvl[lv + 1]; e += nthreads) {
                uint32_t s = 1;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int32_t cq = __ldcg(io.child_q + 4 * size_t(e) + k);
                    if (cq >= 0) s += __ldcg(io.sz + cq);
                }
                __stcg(io.sz + e, s);
            }
            if (!sync()) return false;
        }
        struct PreOut {
            uint32_t* pre;
            __device__ void operator()(int32_t i, uint32_t v) const { __stcg(pre + i, v); }
        };
        for (uint32_t lv = 0; lv < depth; ++lv) {
            for (uint32_t e = s_lvl[lv] + tid; e < s_lvl[lv + 1]; e += nthreads) {
                int32_t cand[4], cq[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    cand[k] = __ldcg(io.cand + 4 * size_t(e) + k);
                    cq[k] = __ldcg(io.child_q + 4 * size_t(e) + k);
                }
                write_node4<NC>(io.n2, cand, cq, __ldcg(pre + e), SizeOf{io.sz}, PreOut{pre}, io.out4, io.map4);
            }
            if (!sync()) return false;
        }
        *total_out = end;
        *depth_out = depth;
        return true;
    } else {
        for (uint32_t e = tid; e < end; e += nthreads) {
            if (inner_children(io, e) != 0u) continue;
            uint32_t cur = e, s = 1u;
            __stcg(io.sz + cur, s);
            for (uint32_t guard = 0;; ++guard) {
                const uint32_t pk = __ldcg(io.par + cur);
                if (pk == kNoParent) break;
                if (guard >= max_levels) {
                    set_err(err, RQ_DERR_QUEUE);
                    break;
                }
                const uint32_t p = pk >> 2;
                const unsigned long long old = atomicAdd(io.acc + p, (1ull << 32) | s);
                if (uint32_t(old >> 32) + 1u < inner_children(io, p)) break;
                s = 1u + uint32_t(old) + s;
                __stcg(io.sz + p, s);
                cur = p;
            }
        }
        if (!sync()) return false;
        // a written node publishes its inner children's positions in `acc`
        // (bit 63 set; phase 2 never sets it), so most walks stop at once
        struct PrePublish {
            unsigned long long* acc;
            __device__ void operator()(int32_t i, uint32_t v) const { __stcg(acc + i, (1ull << 63) | v); }
        };
        for (uint32_t e = tid; e < end; e += nthreads) {
            uint32_t pre = 0, cur = e;
            for (;;) {
                const unsigned long long a = __ldcg(io.acc + cur);
                if (a >> 63) {
                    pre += uint32_t(a);
                    break;
                }
                const uint32_t pk = __ldcg(io.par + cur);
                if (pk == kNoParent) break;  // the root, at 0
                const uint32_t p = pk >> 2, slot = pk & 3u;
                uint32_t off = 1u;
                for (uint32_t j = 0; j < slot; ++j) {
                    const int32_t cq = __ldcg(io.child_q + 4 * size_t(p) + j);
                    if (cq >= 0) off += __ldcg(io.sz + cq);
                }
                pre += off;
                cur = p;
            }
            int32_t cand[4], cq[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                cand[k] = __ldcg(io.cand + 4 * size_t(e) + k);
                cq[k] = __ldcg(io.child_q + 4 * size_t(e) + k);
            }
            write_node4<NC>(io.n2, cand, cq, pre, SizeOf{io.sz}, PrePublish{io.acc}, io.out4, io.map4);
        }
        if (!sync()) return false;
        *total_out = end;
        *depth_out = depth;
        return true;
    }
}

}  // namespace rq
