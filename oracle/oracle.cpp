// oracle.cpp — TEST INFRASTRUCTURE, not product code.
//
// CPU restatement of the reference's BVH build and software traversal path,
// used only as the checker by tests/, __graft_entry__.smoke() and the CPU
// legs of bench.py.  Built to oracle/_build/liboracle.so with
// -ffp-contract=off so every float operation is a single IEEE rounding
// (explicit fmaf where the specification says fused).
//
// Contents (each function cites what it restates):
//   Oracle B — LBVH: prim setup, 30-bit Morton codes, (code, id) sort, Karras
//              2012 hierarchy, <= max_leaf leaves, depth-first emission in the
//              layouts of common/software_bvh.hpp, and the greedy 4-wide
//              collapse of software_bvh.hpp:202-291.
//   Oracle C — fast_bvh_builder.comp:91-257: the RADV image of an implicit
//              4-ary tree over the triangles in input order.
//   Traversals — software_bvh_bvh4.comp:96-195 and software_bvh_lds.comp:86-175
//              as published (reference semantics), plus the engine's own
//              4-wide traversal and RADV-image traversal specification.
//   Ray generators — software_bvh_bvh4.comp:50-94 (PCG procedural rays),
//              visbuf_raycast.comp:15-51 (primary rays, with jitter),
//              tiled_lighting_ra.comp:118-158 (shadow rays), rq_ao.comp:18-94
//              (cosine-hemisphere AO rays).
//
// Parity status: Oracle B and the engine's traversal specification are
// restatements written for this engine (the reference has no LBVH and no CPU
// traversal); they are pinned by the tests against the reference's own
// compiled SoftwareBVH (oracle/_ref) and the golden statistics in the
// reference's results/exp0_ray_stats.csv.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../include/rq.h"

namespace {

// ---------------------------------------------------------------- helpers --

inline float fmin_(float a, float b) { return std::fmin(a, b); }
inline float fmax_(float a, float b) { return std::fmax(a, b); }

struct V3 {
    float x, y, z;
};
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline V3 normalize(V3 v) {
    float len = std::sqrt(dot(v, v));
    return {v.x / len, v.y / len, v.z / len};
}
inline float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Items handed out in chunks of 16..1024, at least 16 chunks per thread
// when n allows, so small batches of heavy items (a pixel's 17 rays) still
// keep every thread busy.
template <class F>
void parallel_for(uint32_t n, int threads, F&& f) {
    if (threads <= 1 || n < 64) {
        for (uint32_t i = 0; i < n; ++i) f(i);
        return;
    }
    const uint32_t chunk = std::max(16u, std::min(1024u, n / (16u * uint32_t(threads))));
    std::atomic<uint32_t> next{0};
    auto worker = [&]() {
        for (;;) {
            uint32_t b = next.fetch_add(chunk);
            if (b >= n) break;
            uint32_t e = std::min(n, b + chunk);
            for (uint32_t i = b; i < e; ++i) f(i);
        }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
}

// Traversal stack without heap traffic: 1024 entries, far above the
// 3*depth+1 a 4-wide traversal can need for any tree the engine accepts.
template <class T>
struct FixedStack {
    T v[1024];
    int n = 0;
    void push_back(const T& x) {
        if (n < 1024) v[n++] = x;
    }
    bool empty() const { return n == 0; }
    T back() const { return v[n - 1]; }
    void pop_back() { --n; }
};

inline V3 load_vertex(const float* pos, uint32_t stride_floats, uint32_t v) {
    const float* p = pos + size_t(v) * stride_floats;
    return {p[0], p[1], p[2]};
}

inline void tri_vertices(const float* pos, uint32_t stride_floats, const uint32_t* idx, uint32_t t,
                         V3& p0, V3& p1, V3& p2) {
    uint32_t i0 = idx ? idx[3 * size_t(t)] : 3 * t;
    uint32_t i1 = idx ? idx[3 * size_t(t) + 1] : 3 * t + 1;
    uint32_t i2 = idx ? idx[3 * size_t(t) + 2] : 3 * t + 2;
    p0 = load_vertex(pos, stride_floats, i0);
    p1 = load_vertex(pos, stride_floats, i1);
    p2 = load_vertex(pos, stride_floats, i2);
}

// ------------------------------------------------------------- Oracle B --

struct Prim {
    float mn[3], mx[3], c[3];
};

// Per-triangle box and centroid exactly as SoftwareBVH::build
// (common/software_bvh.hpp:40-55): centroid = ((p0 + p1) + p2) / 3.0f.
Prim make_prim(V3 p0, V3 p1, V3 p2) {
    Prim p;
    for (int k = 0; k < 3; ++k) {
        float a = comp(p0, k), b = comp(p1, k), c = comp(p2, k);
        p.mn[k] = std::min({a, b, c});
        p.mx[k] = std::max({a, b, c});
        p.c[k] = ((a + b) + c) / 3.0f;
    }
    return p;
}

inline uint32_t expand10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

inline uint32_t quantize(float c, float lo, float scale) {
    float t = (c - lo) * scale;
    if (t >= 1023.0f) return 1023u;
    if (t > 0.0f) return uint32_t(t);
    return 0u;
}

// 30-bit Morton code of each centroid inside the cube spanned by the centroid
// bounds' largest extent (one scale for all three axes).
void morton_codes(const std::vector<Prim>& prims, std::vector<uint32_t>& codes) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (const Prim& p : prims)
        for (int k = 0; k < 3; ++k) {
            lo[k] = fmin_(lo[k], p.c[k]);
            hi[k] = fmax_(hi[k], p.c[k]);
        }
    float ext = fmax_(fmax_(hi[0] - lo[0], hi[1] - lo[1]), hi[2] - lo[2]);
    float scale = ext > 1e-30f ? 1024.0f / ext : 0.0f;
    codes.resize(prims.size());
    for (size_t i = 0; i < prims.size(); ++i) {
        const Prim& p = prims[i];
        codes[i] = expand10(quantize(p.c[0], lo[0], scale)) * 4u +
                   expand10(quantize(p.c[1], lo[1], scale)) * 2u +
                   expand10(quantize(p.c[2], lo[2], scale));
    }
}

inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

struct Karras {
    const std::vector<uint32_t>& k;
    int64_t n;
    int delta(int64_t i, int64_t j) const {
        if (j < 0 || j > n - 1) return -1;
        uint32_t x = k[size_t(i)] ^ k[size_t(j)];
        if (x) return clz32(x);
        return 32 + clz32(uint32_t(i) ^ uint32_t(j));
    }
};

struct KNode {            // Karras internal node
    int64_t lo, hi;       // leaf range, inclusive
    int64_t left, right;  // child indices
    bool left_leaf, right_leaf;
};

// Karras 2012, "Maximizing parallelism in the construction of BVHs, octrees
// and k-d trees", Algorithm for internal node i (sorted keys, ties broken by
// the sorted position).
KNode karras_node(const Karras& K, int64_t i) {
    int d = (K.delta(i, i + 1) - K.delta(i, i - 1)) >= 0 ? 1 : -1;
    int dmin = K.delta(i, i - d);
    int64_t lmax = 2;
    while (K.delta(i, i + lmax * d) > dmin) lmax <<= 1;
    int64_t l = 0;
    for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
        if (K.delta(i, i + (l + t) * d) > dmin) l += t;
    int64_t j = i + l * d;
    int dnode = K.delta(i, j);
    int64_t s = 0, t = l;
    do {
        t = (t + 1) >> 1;
        if (K.delta(i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int64_t gamma = i + s * d + std::min(d, 0);
    KNode kn;
    kn.lo = std::min(i, j);
    kn.hi = std::max(i, j);
    kn.left = gamma;
    kn.left_leaf = kn.lo == gamma;
    kn.right = gamma + 1;
    kn.right_leaf = kn.hi == gamma + 1;
    return kn;
}

struct LbvhState {
    std::vector<Prim> prims;        // original order
    std::vector<uint32_t> codes;    // original order
    std::vector<uint32_t> sorted;   // sorted position -> original id
    std::vector<uint32_t> skeys;    // sorted keys
    std::vector<KNode> inner;
    std::vector<rq_bvh2_node> out;
    uint32_t max_leaf;
};

void union_range(const LbvhState& S, int64_t lo, int64_t hi, float mn[3], float mx[3]) {
    for (int k = 0; k < 3; ++k) {
        mn[k] = INFINITY;
        mx[k] = -INFINITY;
    }
    for (int64_t p = lo; p <= hi; ++p) {
        const Prim& pr = S.prims[S.sorted[size_t(p)]];
        for (int k = 0; k < 3; ++k) {
            mn[k] = fmin_(mn[k], pr.mn[k]);
            mx[k] = fmax_(mx[k], pr.mx[k]);
        }
    }
}

// Depth-first pre-order emission (left child = parent + 1, right child after
// the left subtree, leaves as ~first / count) — the node order of
// SoftwareBVH::recursiveBuild (common/software_bvh.hpp:90-175).
int32_t emit(LbvhState& S, bool is_leaf, int64_t id) {
    int64_t lo, hi;
    if (is_leaf) {
        lo = hi = id;
    } else {
        lo = S.inner[size_t(id)].lo;
        hi = S.inner[size_t(id)].hi;
    }
    int32_t me = int32_t(S.out.size());
    S.out.emplace_back();
    float mn[3], mx[3];
    union_range(S, lo, hi, mn, mx);
    for (int k = 0; k < 3; ++k) {
        S.out[me].aabb_min[k] = mn[k];
        S.out[me].aabb_max[k] = mx[k];
    }
    int64_t cnt = hi - lo + 1;
    if (cnt <= int64_t(S.max_leaf)) {
        S.out[me].left_child = ~int32_t(lo);
        S.out[me].right_child = int32_t(cnt);
        return me;
    }
    const KNode& kn = S.inner[size_t(id)];
    int32_t l = emit(S, kn.left_leaf, kn.left);
    int32_t r = emit(S, kn.right_leaf, kn.right);
    S.out[me].left_child = l;
    S.out[me].right_child = r;
    return me;
}

// ------------------------------------- LBVH with SAH-rebuilt subtrees --
// The LBVH's Karras hierarchy above every node of at most K primitives; each
// such subtree (a contiguous range of the Morton-sorted order) rebuilt top
// down by binned SAH: B bins per axis over the node's centroid bounds (B =
// 16 for nodes of more than kSahSmallNode primitives, 8 for the others), bin
// b = min(B - 1, int((c - cmin) * (B / extent))), split cost
// float(nL) * SA(left) + float(nR) * SA(right) with SA = 2((dx dy + dy dz) + dz dx),
// the smallest cost wins (strict <: the lower axis, then the lower bin, on
// ties), a stable partition of the range; leaves of at most max_leaf
// primitives; the middle of the range where no axis has a centroid extent
// or the subtree is kSahDepthCap levels deep.  Nodes in depth-first pre-order.
constexpr int kSahBinsMax = 16;
constexpr uint32_t kSahSmallNode = 32;
constexpr uint32_t kSahDepthCap = 24;

struct SahState {
    LbvhState* S;
    uint32_t K;
    std::vector<uint32_t> order;  // leaf position -> original primitive
};

inline float sah_area(const float mn[3], const float mx[3]) {
    const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return 2.0f * ((dx * dy + dy * dz) + dz * dx);
}

inline int sah_bin(float c, float cmin, float scale, int bins) {
    const int b = int((c - cmin) * scale);
    return b < bins - 1 ? b : bins - 1;
}

int32_t emit_sah(SahState& T, uint32_t s, uint32_t e, uint32_t depth) {
    LbvhState& S = *T.S;
    const int32_t me = int32_t(S.out.size());
    S.out.emplace_back();
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    float cmn[3] = {INFINITY, INFINITY, INFINITY}, cmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = s; i < e; ++i) {
        const Prim& p = S.prims[T.order[i]];
        for (int k = 0; k < 3; ++k) {
            mn[k] = fmin_(mn[k], p.mn[k]);
            mx[k] = fmax_(mx[k], p.mx[k]);
            cmn[k] = fmin_(cmn[k], p.c[k]);
            cmx[k] = fmax_(cmx[k], p.c[k]);
        }
    }
    for (int k = 0; k < 3; ++k) {
        S.out[me].aabb_min[k] = mn[k];
        S.out[me].aabb_max[k] = mx[k];
    }
    const uint32_t n = e - s;
    if (n <= S.max_leaf) {
        S.out[me].left_child = ~int32_t(s);
        S.out[me].right_child = int32_t(n);
        return me;
    }
    float best = INFINITY, best_scale = 0.0f;
    int best_axis = -1, best_bin = -1;
    uint32_t best_nl = 0;
    const int bins = n > kSahSmallNode ? 16 : 8;
    if (depth < kSahDepthCap) {
        for (int a = 0; a < 3; ++a) {
            const float ext = cmx[a] - cmn[a];
            if (!(ext > 0.0f)) continue;
            const float scale = float(bins) / ext;
            if (!(scale < INFINITY)) continue;  // an extent too small to scale: no split there
            uint32_t cnt[kSahBinsMax] = {};
            float bmn[kSahBinsMax][3], bmx[kSahBinsMax][3];
            for (int b = 0; b < bins; ++b)
                for (int k = 0; k < 3; ++k) {
                    bmn[b][k] = INFINITY;
                    bmx[b][k] = -INFINITY;
                }
            for (uint32_t i = s; i < e; ++i) {
                const Prim& p = S.prims[T.order[i]];
                const int b = sah_bin(p.c[a], cmn[a], scale, bins);
                ++cnt[b];
                for (int k = 0; k < 3; ++k) {
                    bmn[b][k] = fmin_(bmn[b][k], p.mn[k]);
                    bmx[b][k] = fmax_(bmx[b][k], p.mx[k]);
                }
            }
            for (int split = 0; split < bins - 1; ++split) {
                float lmn[3] = {INFINITY, INFINITY, INFINITY}, lmx[3] = {-INFINITY, -INFINITY, -INFINITY};
                float rmn[3] = {INFINITY, INFINITY, INFINITY}, rmx[3] = {-INFINITY, -INFINITY, -INFINITY};
                uint32_t nl = 0, nr = 0;
                for (int b = 0; b < bins; ++b) {
                    float* tmn = b <= split ? lmn : rmn;
                    float* tmx = b <= split ? lmx : rmx;
                    (b <= split ? nl : nr) += cnt[b];
                    for (int k = 0; k < 3; ++k) {
                        tmn[k] = fmin_(tmn[k], bmn[b][k]);
                        tmx[k] = fmax_(tmx[k], bmx[b][k]);
                    }
                }
                const float cost = float(nl) * sah_area(lmn, lmx) + float(nr) * sah_area(rmn, rmx);
                if (cost < best) {
                    best = cost;
                    best_axis = a;
                    best_bin = split;
                    best_scale = scale;
                    best_nl = nl;
                }
            }
        }
    }
    uint32_t mid;
    if (best_axis < 0) {
        mid = s + n / 2;
    } else {
        std::vector<uint32_t> left, right;
        for (uint32_t i = s; i < e; ++i) {
            const uint32_t id = T.order[i];
            (sah_bin(S.prims[id].c[best_axis], cmn[best_axis], best_scale, bins) <= best_bin ? left : right).push_back(id);
        }
        std::copy(left.begin(), left.end(), T.order.begin() + s);
        std::copy(right.begin(), right.end(), T.order.begin() + s + left.size());
        mid = s + best_nl;
    }
    const int32_t l = emit_sah(T, s, mid, depth + 1);
    const int32_t r = emit_sah(T, mid, e, depth + 1);
    S.out[me].left_child = l;
    S.out[me].right_child = r;
    return me;
}

int32_t emit_top(SahState& T, bool is_leaf, int64_t id) {
    LbvhState& S = *T.S;
    const int64_t lo = is_leaf ? id : S.inner[size_t(id)].lo;
    const int64_t hi = is_leaf ? id : S.inner[size_t(id)].hi;
    if (uint64_t(hi - lo + 1) <= T.K) return emit_sah(T, uint32_t(lo), uint32_t(hi + 1), 0);
    const int32_t me = int32_t(S.out.size());
    S.out.emplace_back();
    float mn[3], mx[3];
    union_range(S, lo, hi, mn, mx);
    for (int k = 0; k < 3; ++k) {
        S.out[me].aabb_min[k] = mn[k];
        S.out[me].aabb_max[k] = mx[k];
    }
    const KNode& kn = S.inner[size_t(id)];
    const int32_t l = emit_top(T, kn.left_leaf, kn.left);
    const int32_t r = emit_top(T, kn.right_leaf, kn.right);
    S.out[me].left_child = l;
    S.out[me].right_child = r;
    return me;
}

// Greedy 4-wide collapse: restates SoftwareBVH4::collapse
// (common/software_bvh.hpp:202-291) — open the inner candidate with the
// largest surface area (strict >, first wins) until four candidates, emit in
// depth-first pre-order, zero-filled empty slots.
int32_t collapse4(const rq_bvh2_node* n2, int32_t idx, std::vector<rq_bvh4_node>& out, uint32_t depth,
                  uint32_t* max_depth) {
    if (depth > *max_depth) *max_depth = depth;
    const rq_bvh2_node& node = n2[idx];
    if (node.left_child < 0) {
        int32_t o = int32_t(out.size());
        out.emplace_back();
        std::memset(&out[o], 0, sizeof(rq_bvh4_node));
        out[o].min_x[0] = node.aabb_min[0];
        out[o].max_x[0] = node.aabb_max[0];
        out[o].min_y[0] = node.aabb_min[1];
        out[o].max_y[0] = node.aabb_max[1];
        out[o].min_z[0] = node.aabb_min[2];
        out[o].max_z[0] = node.aabb_max[2];
        out[o].child_index[0] = node.left_child;
        out[o].child_count[0] = node.right_child;
        return o;
    }
    int32_t cand[4];
    int nc = 2;
    cand[0] = node.left_child;
    cand[1] = node.right_child;
    while (nc < 4) {
        int best = -1;
        float best_sa = -1.0f;
        for (int i = 0; i < nc; ++i) {
            const rq_bvh2_node& c = n2[cand[i]];
            if (c.left_child >= 0) {
                float dx = c.aabb_max[0] - c.aabb_min[0];
                float dy = c.aabb_max[1] - c.aabb_min[1];
                float dz = c.aabb_max[2] - c.aabb_min[2];
                float sa = 2.0f * ((dx * dy + dy * dz) + dz * dx);
                if (sa > best_sa) {
                    best_sa = sa;
                    best = i;
                }
            }
        }
        if (best < 0) break;
        int32_t e = cand[best];
        cand[best] = n2[e].left_child;
        cand[nc++] = n2[e].right_child;
    }
    int32_t o = int32_t(out.size());
    out.emplace_back();
    rq_bvh4_node tmp;
    std::memset(&tmp, 0, sizeof(tmp));
    for (int i = 0; i < nc; ++i) {
        const rq_bvh2_node& c = n2[cand[i]];
        tmp.min_x[i] = c.aabb_min[0];
        tmp.max_x[i] = c.aabb_max[0];
        tmp.min_y[i] = c.aabb_min[1];
        tmp.max_y[i] = c.aabb_max[1];
        tmp.min_z[i] = c.aabb_min[2];
        tmp.max_z[i] = c.aabb_max[2];
        if (c.left_child < 0) {
            tmp.child_index[i] = c.left_child;
            tmp.child_count[i] = c.right_child;
        } else {
            tmp.child_count[i] = -1;
        }
    }
    for (int i = 0; i < nc; ++i)
        if (n2[cand[i]].left_child >= 0) tmp.child_index[i] = collapse4(n2, cand[i], out, depth + 1, max_depth);
    out[o] = tmp;
    return o;
}

// ------------------------------------------------------------- Oracle C --

const uint32_t kQNaN = 0x7fc00000u;

inline float bits_f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// ------------------------------------------------------------- traversal --

// Möller–Trumbore as written in software_bvh_bvh4.comp:166-178 (|a| < eps
// rejected, u,v in [0,1], u+v <= 1).  Returns false on reject, else t.
inline bool mt_test(V3 o, V3 d, V3 v0, V3 v1, V3 v2, float eps, float& t, float& u, float& v) {
    V3 e1 = sub(v1, v0);
    V3 e2 = sub(v2, v0);
    V3 h = cross(d, e2);
    float a = dot(e1, h);
    if (std::fabs(a) < eps) return false;
    float f = 1.0f / a;
    V3 s = sub(o, v0);
    u = f * dot(s, h);
    if (u < 0.0f || u > 1.0f) return false;
    V3 q = cross(s, e1);
    v = f * dot(d, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    t = f * dot(e2, q);
    return true;
}

// Per-ray constants of the watertight test (Woop, Benthin, Wald 2013).
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

inline WtRay wt_setup(V3 d) {
    WtRay w;
    float ad[3] = {std::fabs(d.x), std::fabs(d.y), std::fabs(d.z)};
    int kz = 0;
    if (ad[1] > ad[kz]) kz = 1;
    if (ad[2] > ad[kz]) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (comp(d, kz) < 0.0f) std::swap(kx, ky);
    w.kx = kx;
    w.ky = ky;
    w.kz = kz;
    w.sx = comp(d, kx) / comp(d, kz);
    w.sy = comp(d, ky) / comp(d, kz);
    w.sz = 1.0f / comp(d, kz);
    return w;
}

// Watertight test: edge functions in plain float products (so a shared edge
// evaluates to exact negations), double recomputation when any is 0.0, t by
// one IEEE division.  u, v are the weights of v1 and v2.
inline bool wt_test(const WtRay& w, V3 o, V3 v0, V3 v1, V3 v2, float& t, float& u, float& v) {
    V3 A = sub(v0, o), B = sub(v1, o), C = sub(v2, o);
    float Az0 = comp(A, w.kz), Bz0 = comp(B, w.kz), Cz0 = comp(C, w.kz);
    float Ax = std::fmaf(-w.sx, Az0, comp(A, w.kx));
    float Ay = std::fmaf(-w.sy, Az0, comp(A, w.ky));
    float Bx = std::fmaf(-w.sx, Bz0, comp(B, w.kx));
    float By = std::fmaf(-w.sy, Bz0, comp(B, w.ky));
    float Cx = std::fmaf(-w.sx, Cz0, comp(C, w.kx));
    float Cy = std::fmaf(-w.sy, Cz0, comp(C, w.ky));
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = float(double(Cx) * double(By) - double(Cy) * double(Bx));
        V = float(double(Ax) * double(Cy) - double(Ay) * double(Cx));
        W = float(double(Bx) * double(Ay) - double(By) * double(Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = (U + V) + W;
    if (det == 0.0f) return false;
    float Az = w.sz * Az0, Bz = w.sz * Bz0, Cz = w.sz * Cz0;
    float T = (U * Az + V * Bz) + W * Cz;
    t = T / det;
    u = V / det;
    v = W / det;
    return true;
}

const float kTwoPow100 = 1.2676506002282294e30f;  // 2^100
const float kTwoPowM100 = 7.888609052210118e-31f;  // 2^-100
const float kFarScale = 1.00000095367431640625f;   // 1 + 2^-20

inline float safe_inv(float d) {
    if (std::fabs(d) < kTwoPowM100) return std::copysign(kTwoPow100, d);
    return 1.0f / d;
}

// Slab test of the engine's traversal: fused (b*inv - o*inv), entry clamped
// by tmin, exit by the current best, exit widened by 2^-20 relative.
inline bool slab(const float inv[3], const float oinv[3], float tmin, float best, float mnx, float mxx,
                 float mny, float mxy, float mnz, float mxz, float& tn) {
    float tx0 = std::fmaf(mnx, inv[0], -oinv[0]), tx1 = std::fmaf(mxx, inv[0], -oinv[0]);
    float ty0 = std::fmaf(mny, inv[1], -oinv[1]), ty1 = std::fmaf(mxy, inv[1], -oinv[1]);
    float tz0 = std::fmaf(mnz, inv[2], -oinv[2]), tz1 = std::fmaf(mxz, inv[2], -oinv[2]);
    float a = fmax_(fmax_(fmin_(tx0, tx1), fmin_(ty0, ty1)), fmax_(fmin_(tz0, tz1), tmin));
    float b = fmin_(fmin_(fmax_(tx0, tx1), fmax_(ty0, ty1)), fmin_(fmax_(tz0, tz1), best));
    tn = a;
    return a <= b * kFarScale;
}

// The engine's 4-wide slab test (rq_device.cuh box4_nf): each axis's near
// and far plane picked by the sign bit of inv (the max plane when inv is
// negative), entry max(near_x, near_y, near_z, tmin), exit
// min(far_x, far_y, far_z, best).  For boxes with min <= max this equals
// slab() above; boxes with min > max on an axis are empty.
inline bool slab4(const float inv[3], const float oinv[3], float tmin, float best, const rq_bvh4_node& n, int k,
                  float& tn) {
    const float* lo[3] = {n.min_x, n.min_y, n.min_z};
    const float* hi[3] = {n.max_x, n.max_y, n.max_z};
    float tnear[3], tfar[3];
    for (int a = 0; a < 3; ++a) {
        const bool neg = std::signbit(inv[a]);
        tnear[a] = std::fmaf((neg ? hi[a] : lo[a])[k], inv[a], -oinv[a]);
        tfar[a] = std::fmaf((neg ? lo[a] : hi[a])[k], inv[a], -oinv[a]);
    }
    const float a = fmax_(fmax_(fmax_(tnear[0], tnear[1]), tnear[2]), tmin);
    const float b = fmin_(fmin_(fmin_(tfar[0], tfar[1]), tfar[2]), best);
    tn = a;
    return a <= b * kFarScale;
}

struct TraceOut {
    bool hit;
    float t;
    uint32_t prim;  // leaf-order index (or RADV triangle node offset)
    float u, v;
    uint32_t boxes, tris;
};

// The engine's 4-wide traversal (rq_trace).  Stack of entries; inner nodes
// and leaf children are both pushed.  Closest hit: hit children sorted by
// entry distance (ties by slot), pushed far-first.  Any hit: hit children
// pushed from slot 3 down to slot 0 (slot 0 on top), traversal stops at the
// first accepted triangle.  A leaf tests its triangles in order.
TraceOut trace_bvh4(const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_ray& r, uint32_t flags) {
    const bool any = flags & 1u;
    const bool mt = flags & 2u;
    V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
    float inv[3] = {safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
    float oinv[3] = {o.x * inv[0], o.y * inv[1], o.z * inv[2]};
    WtRay w = wt_setup(d);
    float tmin = r.tmin, best = r.tmax;
    TraceOut res{false, -1.0f, 0xffffffffu, 0.0f, 0.0f, 0, 0};
    struct Entry {
        int32_t idx;   // node index, or first prim for a leaf
        int32_t cnt;   // -1 inner, else prim count
    };
    FixedStack<Entry> st;
    st.push_back({0, -1});
    while (!st.empty()) {
        Entry e = st.back();
        st.pop_back();
        if (e.cnt < 0) {
            const rq_bvh4_node& n = nodes[e.idx];
            res.boxes += 4;
            Entry hc[4];
            float ht[4];
            int nh = 0;
            for (int k = 0; k < 4; ++k) {
                if (n.child_count[k] == 0) continue;
                float tn;
                if (slab4(inv, oinv, tmin, best, n, k, tn)) {
                    Entry c;
                    if (n.child_count[k] < 0) {
                        c = {n.child_index[k], -1};
                    } else {
                        c = {~n.child_index[k], n.child_count[k]};
                    }
                    // insertion keeps ascending distance, stable by slot
                    int pos = nh;
                    if (!any)
                        while (pos > 0 && ht[pos - 1] > tn) {
                            hc[pos] = hc[pos - 1];
                            ht[pos] = ht[pos - 1];
                            --pos;
                        }
                    hc[pos] = c;
                    ht[pos] = tn;
                    ++nh;
                }
            }
            for (int i = nh - 1; i >= 0; --i) st.push_back(hc[i]);
        } else {
            for (int32_t p = 0; p < e.cnt; ++p) {
                uint32_t pi = uint32_t(e.idx + p);
                const rq_triangle& tr = tris[pi];
                V3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]},
                    v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                res.tris += 1;
                float t, u, v;
                bool ok = mt ? mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v) : wt_test(w, o, v0, v1, v2, t, u, v);
                if (ok && t >= tmin && t < best) {
                    best = t;
                    res.hit = true;
                    res.t = t;
                    res.prim = pi;
                    res.u = u;
                    res.v = v;
                    if (any) return res;
                }
            }
        }
    }
    return res;
}

// RADV image traversal (rq_trace_radv): same ordering rules; a Box32 child is
// either another Box32 (type 5) or a 64-B triangle node (type 0).
TraceOut trace_radv(const uint8_t* img, const rq_ray& r, uint32_t flags) {
    const bool any = flags & 1u;
    const bool mt = flags & 2u;
    V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
    float inv[3] = {safe_inv(d.x), safe_inv(d.y), safe_inv(d.z)};
    float oinv[3] = {o.x * inv[0], o.y * inv[1], o.z * inv[2]};
    WtRay w = wt_setup(d);
    float tmin = r.tmin, best = r.tmax;
    TraceOut res{false, -1.0f, 0xffffffffu, 0.0f, 0.0f, 0, 0};
    const uint8_t* base = img + RQ_RADV_BVH_OFFSET;
    FixedStack<uint32_t> st;
    st.push_back(RQ_RADV_NODE_BOX32);
    while (!st.empty()) {
        uint32_t id = st.back();
        st.pop_back();
        uint32_t type = id & 7u;
        const uint8_t* p = base + (size_t(id & ~7u) << 3);
        if (type == RQ_RADV_NODE_BOX32) {
            rq_radv_box32 b;
            std::memcpy(&b, p, sizeof(b));
            res.boxes += 4;
            uint32_t hc[4];
            float ht[4];
            int nh = 0;
            for (int k = 0; k < 4; ++k) {
                if (b.children[k] == RQ_RADV_INVALID_NODE) continue;
                const float* c = b.coords[k];
                float tn;
                if (slab(inv, oinv, tmin, best, c[0], c[3], c[1], c[4], c[2], c[5], tn)) {
                    int pos = nh;
                    if (!any)
                        while (pos > 0 && ht[pos - 1] > tn) {
                            hc[pos] = hc[pos - 1];
                            ht[pos] = ht[pos - 1];
                            --pos;
                        }
                    hc[pos] = b.children[k];
                    ht[pos] = tn;
                    ++nh;
                }
            }
            for (int i = nh - 1; i >= 0; --i) st.push_back(hc[i]);
        } else if (type == RQ_RADV_NODE_TRIANGLE) {
            rq_radv_tri tn;
            std::memcpy(&tn, p, sizeof(tn));
            V3 v0{tn.coords[0][0], tn.coords[0][1], tn.coords[0][2]};
            V3 v1{tn.coords[1][0], tn.coords[1][1], tn.coords[1][2]};
            V3 v2{tn.coords[2][0], tn.coords[2][1], tn.coords[2][2]};
            res.tris += 1;
            float t, u, v;
            bool ok = mt ? mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v) : wt_test(w, o, v0, v1, v2, t, u, v);
            if (ok && t >= tmin && t < best) {
                best = t;
                res.hit = true;
                res.t = t;
                res.prim = tn.triangle_id;
                res.u = u;
                res.v = v;
                if (any) return res;
            }
        }
    }
    return res;
}

// ------------------------------------------------------------ ray makers --

inline uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
const float kInv2Pow32 = 2.3283064365386963e-10f;  // 1/4294967295.0 evaluated in float = 2^-32
inline float hash_float(uint32_t seed) { return float(pcg_hash(seed)) * kInv2Pow32; }

// One-at-a-time style hash of rq_ao.comp:18-25.
inline uint32_t ao_hash(uint32_t x) {
    x += (x << 10u);
    x ^= (x >> 6u);
    x += (x << 3u);
    x ^= (x >> 11u);
    x += (x << 15u);
    return x;
}

// sin/cos for the AO hemisphere: Cody–Waite reduction by pi/2 in three
// parts and Taylor polynomials (coefficients 1/n!) on [-pi/4, pi/4], all
// with explicit fused multiply-adds, so the device code can match bit for bit.
inline void sincos_taylor(float x, float* s, float* c) {
    float n = std::floor(std::fmaf(x, 0x1.45f306p-1f, 0.5f));
    float r = std::fmaf(-n, 0x1.921fb6p+0f, x);
    r = std::fmaf(-n, -0x1.777a5cp-25f, r);
    r = std::fmaf(-n, -0x1.ee59dap-50f, r);
    float r2 = r * r;
    float ps = std::fmaf(r2, 0x1.71de3ap-19f, -0x1.a01a02p-13f);
    ps = std::fmaf(r2, ps, 0x1.111112p-7f);
    ps = std::fmaf(r2, ps, -0x1.555556p-3f);
    ps = std::fmaf(r2 * r, ps, r);
    float pc = std::fmaf(r2, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = std::fmaf(r2, pc, -0x1.6c16c2p-10f);
    pc = std::fmaf(r2, pc, 0x1.555556p-5f);
    pc = std::fmaf(r2, pc, -0.5f);
    pc = std::fmaf(r2, pc, 1.0f);
    int q = int(int64_t(n) & 3);
    float sv = q == 0 ? ps : (q == 1 ? pc : (q == 2 ? -ps : -pc));
    float cv = q == 0 ? pc : (q == 1 ? -ps : (q == 2 ? -pc : ps));
    *s = sv;
    *c = cv;
}

// Matrix (column-major, GLSL convention) times (x, y, z, w).
inline void mat4_mul(const float* m, const float in[4], float out[4]) {
    for (int r = 0; r < 4; ++r)
        out[r] = ((m[0 * 4 + r] * in[0] + m[1 * 4 + r] * in[1]) + m[2 * 4 + r] * in[2]) + m[3 * 4 + r] * in[3];
}

}  // namespace

// =================================================================== C ABI

extern "C" {

// Oracle B, stage by stage.  pos: vertex floats with stride_floats between
// vertices; idx may be NULL (non-indexed).  Outputs sized by the caller:
// codes/sorted/perm: n; nodes2: 2n; nodes4: max(1, n); tris: n.
// Returns the node counts through n2/n4 and the 4-wide depth through depth4.
int orc_lbvh_build(const float* pos, uint32_t stride_floats, const uint32_t* idx, uint32_t n,
                   uint32_t max_leaf, uint32_t* codes_out, uint32_t* sorted_out, rq_bvh2_node* nodes2,
                   uint32_t* n2, rq_triangle* tris, rq_bvh4_node* nodes4, uint32_t* n4, uint32_t* depth4) {
    if (n == 0 || max_leaf == 0) return 1;
    LbvhState S;
    S.max_leaf = max_leaf;
    S.prims.resize(n);
    for (uint32_t t = 0; t < n; ++t) {
        V3 p0, p1, p2;
        tri_vertices(pos, stride_floats, idx, t, p0, p1, p2);
        S.prims[t] = make_prim(p0, p1, p2);
    }
    morton_codes(S.prims, S.codes);
    S.sorted.resize(n);
    for (uint32_t i = 0; i < n; ++i) S.sorted[i] = i;
    std::sort(S.sorted.begin(), S.sorted.end(), [&](uint32_t a, uint32_t b) {
        return S.codes[a] != S.codes[b] ? S.codes[a] < S.codes[b] : a < b;
    });
    S.skeys.resize(n);
    for (uint32_t i = 0; i < n; ++i) S.skeys[i] = S.codes[S.sorted[i]];
    if (codes_out) std::memcpy(codes_out, S.codes.data(), 4ull * n);
    if (sorted_out) std::memcpy(sorted_out, S.sorted.data(), 4ull * n);
    Karras K{S.skeys, int64_t(n)};
    if (n >= 2) {
        S.inner.resize(n - 1);
        for (uint32_t i = 0; i + 1 < n; ++i) S.inner[i] = karras_node(K, i);
    }
    S.out.reserve(2ull * n);
    if (n == 1)
        emit(S, true, 0);
    else
        emit(S, false, 0);
    *n2 = uint32_t(S.out.size());
    if (nodes2) std::memcpy(nodes2, S.out.data(), sizeof(rq_bvh2_node) * S.out.size());
    if (tris) {
        for (uint32_t k = 0; k < n; ++k) {
            V3 p0, p1, p2;
            tri_vertices(pos, stride_floats, idx, S.sorted[k], p0, p1, p2);
            rq_triangle tr;
            tr.v0[0] = p0.x; tr.v0[1] = p0.y; tr.v0[2] = p0.z; tr.v0[3] = 0.0f;
            tr.v1[0] = p1.x; tr.v1[1] = p1.y; tr.v1[2] = p1.z; tr.v1[3] = 0.0f;
            tr.v2[0] = p2.x; tr.v2[1] = p2.y; tr.v2[2] = p2.z; tr.v2[3] = 0.0f;
            tris[k] = tr;
        }
    }
    if (nodes4 || n4) {
        std::vector<rq_bvh4_node> out4;
        uint32_t md = 0;
        collapse4(S.out.data(), 0, out4, 1, &md);
        if (n4) *n4 = uint32_t(out4.size());
        if (depth4) *depth4 = md;
        if (nodes4) std::memcpy(nodes4, out4.data(), sizeof(rq_bvh4_node) * out4.size());
    }
    return 0;
}

// LBVH with SAH-rebuilt subtrees of at most `sah_max` primitives (see
// emit_sah).  Codes and sort as orc_lbvh_build; perm_out[k] = the original
// triangle at leaf position k (the sort permutation, permuted inside each
// rebuilt subtree).
int orc_lbvh_sah_build(const float* pos, uint32_t stride_floats, const uint32_t* idx, uint32_t n, uint32_t max_leaf,
                       uint32_t sah_max, uint32_t* codes_out, uint32_t* sorted_out, rq_bvh2_node* nodes2, uint32_t* n2,
                       rq_triangle* tris, uint32_t* perm_out, rq_bvh4_node* nodes4, uint32_t* n4, uint32_t* depth4) {
    if (n == 0 || max_leaf == 0 || sah_max < max_leaf) return 1;
    LbvhState S;
    S.max_leaf = max_leaf;
    S.prims.resize(n);
    for (uint32_t t = 0; t < n; ++t) {
        V3 p0, p1, p2;
        tri_vertices(pos, stride_floats, idx, t, p0, p1, p2);
        S.prims[t] = make_prim(p0, p1, p2);
    }
    morton_codes(S.prims, S.codes);
    S.sorted.resize(n);
    for (uint32_t i = 0; i < n; ++i) S.sorted[i] = i;
    std::sort(S.sorted.begin(), S.sorted.end(), [&](uint32_t a, uint32_t b) {
        return S.codes[a] != S.codes[b] ? S.codes[a] < S.codes[b] : a < b;
    });
    S.skeys.resize(n);
    for (uint32_t i = 0; i < n; ++i) S.skeys[i] = S.codes[S.sorted[i]];
    if (codes_out) std::memcpy(codes_out, S.codes.data(), 4ull * n);
    if (sorted_out) std::memcpy(sorted_out, S.sorted.data(), 4ull * n);
    Karras K{S.skeys, int64_t(n)};
    if (n >= 2) {
        S.inner.resize(n - 1);
        for (uint32_t i = 0; i + 1 < n; ++i) S.inner[i] = karras_node(K, i);
    }
    SahState T{&S, sah_max, S.sorted};
    S.out.reserve(2ull * n);
    emit_top(T, n == 1, 0);
    *n2 = uint32_t(S.out.size());
    if (nodes2) std::memcpy(nodes2, S.out.data(), sizeof(rq_bvh2_node) * S.out.size());
    if (perm_out) std::memcpy(perm_out, T.order.data(), 4ull * n);
    if (tris) {
        for (uint32_t k = 0; k < n; ++k) {
            V3 p0, p1, p2;
            tri_vertices(pos, stride_floats, idx, T.order[k], p0, p1, p2);
            tris[k] = rq_triangle{{p0.x, p0.y, p0.z, 0.0f}, {p1.x, p1.y, p1.z, 0.0f}, {p2.x, p2.y, p2.z, 0.0f}};
        }
    }
    if (nodes4 || n4) {
        std::vector<rq_bvh4_node> out4;
        uint32_t md = 0;
        collapse4(S.out.data(), 0, out4, 1, &md);
        if (n4) *n4 = uint32_t(out4.size());
        if (depth4) *depth4 = md;
        if (nodes4) std::memcpy(nodes4, out4.data(), sizeof(rq_bvh4_node) * out4.size());
    }
    return 0;
}

// The greedy collapse alone, on any binary BVH in the GpuBvhNode layout.
int orc_collapse4(const rq_bvh2_node* nodes2, uint32_t n2, rq_bvh4_node* nodes4, uint32_t* n4, uint32_t* depth4) {
    if (n2 == 0) {
        *n4 = 0;
        return 0;
    }
    std::vector<rq_bvh4_node> out4;
    uint32_t md = 0;
    collapse4(nodes2, 0, out4, 1, &md);
    *n4 = uint32_t(out4.size());
    if (depth4) *depth4 = md;
    if (nodes4) std::memcpy(nodes4, out4.data(), sizeof(rq_bvh4_node) * out4.size());
    return 0;
}

// Oracle C: fast_bvh_builder.comp:91-257 for any n.  `img` must hold
// 192 + 128*boxes + 64*n bytes; bytes the shader never writes (136..191
// except the two pre-root dwords) are written as 0.
int orc_radv_build(const float* tri9, uint32_t n, uint8_t* img) {
    if (n == 0) return 1;
    std::vector<uint32_t> counts{(n + 3) / 4};
    while (counts.back() > 1) counts.push_back((counts.back() + 3) / 4);
    std::reverse(counts.begin(), counts.end());
    uint32_t levels = uint32_t(counts.size());
    std::vector<uint32_t> offs(levels);
    uint32_t total = 0;
    for (uint32_t l = 0; l < levels; ++l) {
        offs[l] = total;
        total += counts[l];
    }
    uint64_t size = 192ull + 128ull * total + 64ull * n;
    std::memset(img, 0, size);
    std::vector<float> bmin(3ull * total), bmax(3ull * total);
    uint8_t* boxes = img + 192;
    uint8_t* trin = img + 192 + 128ull * total;
    float qnan = bits_f(kQNaN);
    // leaf boxes over four consecutive input triangles
    uint32_t leaf_off = offs[levels - 1], leaf_cnt = counts[levels - 1];
    for (uint32_t t = 0; t < leaf_cnt; ++t) {
        rq_radv_box32 b;
        std::memset(&b, 0, sizeof(b));
        float umin[3] = {1e30f, 1e30f, 1e30f}, umax[3] = {-1e30f, -1e30f, -1e30f};
        for (uint32_t c = 0; c < 4; ++c) {
            uint32_t ti = 4 * t + c;
            if (ti < n) {
                const float* v = tri9 + 9ull * ti;
                rq_radv_tri tn;
                std::memset(&tn, 0, sizeof(tn));
                for (int a = 0; a < 3; ++a)
                    for (int k = 0; k < 3; ++k) tn.coords[a][k] = v[3 * a + k];
                tn.triangle_id = ti;
                tn.geometry_id_and_flags = RQ_RADV_GEOMETRY_OPAQUE;
                tn.id = RQ_RADV_BARYCENTRICS_CONTROL_DEFAULT;
                std::memcpy(trin + 64ull * ti, &tn, 64);
                uint32_t rel = total * 128u + ti * 64u;
                b.children[c] = (rel >> 3) | RQ_RADV_NODE_TRIANGLE;
                for (int k = 0; k < 3; ++k) {
                    float mn = fmin_(v[k], fmin_(v[3 + k], v[6 + k]));
                    float mx = fmax_(v[k], fmax_(v[3 + k], v[6 + k]));
                    b.coords[c][k] = mn;
                    b.coords[c][3 + k] = mx;
                    umin[k] = fmin_(umin[k], mn);
                    umax[k] = fmax_(umax[k], mx);
                }
            } else {
                b.children[c] = RQ_RADV_INVALID_NODE;
                for (int k = 0; k < 6; ++k) b.coords[c][k] = qnan;
            }
        }
        std::memcpy(boxes + 128ull * (leaf_off + t), &b, 128);
        for (int k = 0; k < 3; ++k) {
            bmin[3ull * (leaf_off + t) + k] = umin[k];
            bmax[3ull * (leaf_off + t) + k] = umax[k];
        }
    }
    for (int l = int(levels) - 2; l >= 0; --l) {
        uint32_t cnt = counts[l], off = offs[l], coff = offs[l + 1], ccnt = counts[l + 1];
        for (uint32_t t = 0; t < cnt; ++t) {
            rq_radv_box32 b;
            std::memset(&b, 0, sizeof(b));
            float umin[3] = {1e30f, 1e30f, 1e30f}, umax[3] = {-1e30f, -1e30f, -1e30f};
            for (uint32_t c = 0; c < 4; ++c) {
                uint32_t cl = 4 * t + c;
                if (cl < ccnt) {
                    uint32_t cg = coff + cl;
                    b.children[c] = ((cg * 128u) >> 3) | RQ_RADV_NODE_BOX32;
                    for (int k = 0; k < 3; ++k) {
                        b.coords[c][k] = bmin[3ull * cg + k];
                        b.coords[c][3 + k] = bmax[3ull * cg + k];
                        umin[k] = fmin_(umin[k], bmin[3ull * cg + k]);
                        umax[k] = fmax_(umax[k], bmax[3ull * cg + k]);
                    }
                } else {
                    b.children[c] = RQ_RADV_INVALID_NODE;
                    for (int k = 0; k < 6; ++k) b.coords[c][k] = qnan;
                }
            }
            std::memcpy(boxes + 128ull * (off + t), &b, 128);
            for (int k = 0; k < 3; ++k) {
                bmin[3ull * (off + t) + k] = umin[k];
                bmax[3ull * (off + t) + k] = umax[k];
            }
        }
    }
    rq_radv_header h;
    std::memset(&h, 0, sizeof(h));
    h.bvh_offset = 192;
    for (int k = 0; k < 3; ++k) {
        h.aabb_min[k] = bmin[k];
        h.aabb_max[k] = bmax[k];
    }
    h.update_dispatch_size[0] = 8;
    h.update_dispatch_size[1] = 1;
    h.update_dispatch_size[2] = 1;
    h.compacted_size = size;
    h.serialization_size = size + 128;
    h.copy_dispatch_size[0] = 1;
    h.copy_dispatch_size[1] = 1;
    h.copy_dispatch_size[2] = 1;
    h.size = size;
    h.geometry_count = 1;
    h.leaf_nodes_offset = 192ull + 128ull * total;
    h.primitive_count = n;
    h.build_flags = 4;
    h.type = 1;
    std::memcpy(img, &h, sizeof(h));
    uint32_t five = 5, inval = 0xffffffffu;
    std::memcpy(img + 180, &five, 4);
    std::memcpy(img + 188, &inval, 4);
    return 0;
}

// Reference semantics of software_bvh_bvh4.comp:96-195 on explicit rays
// (ray tmin/tmax replace the shader's constants 0.01 / 1000).  Hit IDs are
// leaf-order indices (:181).  The shader's 24-entry stack drops a push that
// does not fit (:185); dropped[i] (may be NULL) counts them per ray, so a
// miss caused by a dropped subtree can be told from a geometric one.
void orc_trace_ref_bvh4(const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_ray* rays, uint32_t n,
                        rq_ray_stats* stats, rq_hit* hits, uint32_t* dropped, int threads) {
    parallel_for(n, threads, [&](uint32_t idx) {
        const rq_ray& r = rays[idx];
        V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
        V3 inv{std::fabs(d.x) > 1e-6f ? 1.0f / d.x : 1e6f, std::fabs(d.y) > 1e-6f ? 1.0f / d.y : 1e6f,
               std::fabs(d.z) > 1e-6f ? 1.0f / d.z : 1e6f};
        float tmin = r.tmin, hitT = r.tmax;
        int hitPrim = -1;
        uint32_t boxTests = 0, triTests = 0;
        int32_t stack[24];
        stack[0] = 0;
        int ptr = 1;
        uint32_t drops = 0;
        while (ptr > 0) {
            const rq_bvh4_node& nd = nodes[stack[--ptr]];
            boxTests += 4;
            float tEntry[4], tExit[4];
            for (int k = 0; k < 4; ++k) {
                float t0x = (nd.min_x[k] - o.x) * inv.x, t1x = (nd.max_x[k] - o.x) * inv.x;
                float t0y = (nd.min_y[k] - o.y) * inv.y, t1y = (nd.max_y[k] - o.y) * inv.y;
                float t0z = (nd.min_z[k] - o.z) * inv.z, t1z = (nd.max_z[k] - o.z) * inv.z;
                float tminX = fmin_(t0x, t1x), tmaxX = fmax_(t0x, t1x);
                float tminY = fmin_(t0y, t1y), tmaxY = fmax_(t0y, t1y);
                float tminZ = fmin_(t0z, t1z), tmaxZ = fmax_(t0z, t1z);
                tEntry[k] = fmax_(fmax_(tminX, tminY), fmax_(tminZ, tmin));
                tExit[k] = fmin_(fmin_(tmaxX, tmaxY), fmin_(tmaxZ, hitT));
            }
            int slot[4];
            float ht[4];
            int hc = 0;
            for (int k = 0; k < 4; ++k)
                if (nd.child_count[k] != 0 && tExit[k] >= tEntry[k]) {
                    slot[hc] = k;
                    ht[hc] = tEntry[k];
                    ++hc;
                }
            if (hc == 0) continue;
            for (int i = 0; i < hc - 1; ++i)
                for (int j = i + 1; j < hc; ++j)
                    if (ht[i] < ht[j]) {
                        std::swap(ht[i], ht[j]);
                        std::swap(slot[i], slot[j]);
                    }
            for (int i = 0; i < hc; ++i) {
                int k = slot[i];
                if (nd.child_count[k] > 0) {
                    uint32_t first = uint32_t(~nd.child_index[k]);
                    uint32_t cnt = uint32_t(nd.child_count[k]);
                    triTests += cnt;
                    for (uint32_t p = 0; p < cnt; ++p) {
                        const rq_triangle& tr = tris[first + p];
                        V3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]},
                            v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                        float t, u, v;
                        if (!mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v)) continue;
                        if (t >= tmin && t < hitT) {
                            hitT = t;
                            hitPrim = int(first + p);
                        }
                    }
                } else if (nd.child_count[k] < 0) {
                    if (ptr < 24)
                        stack[ptr++] = nd.child_index[k];
                    else
                        ++drops;
                }
            }
        }
        if (dropped) dropped[idx] = drops;
        if (stats) stats[idx] = {hitPrim >= 0 ? 1u : 0u, boxTests, triTests, 0u};
        if (hits) {
            if (hitPrim >= 0)
                hits[idx] = {1u, hitT, 0u, uint32_t(hitPrim)};
            else
                hits[idx] = {0u, -1.0f, 0xffffffffu, 0xffffffffu};
        }
    });
}

// Reference semantics of software_bvh_lds.comp:86-175 (t_eps 0.001) and
// software_bvh_procedural.comp (t_eps 0.01) on explicit rays: root box test
// against the running closest t, children tested from the parent, front-to-
// back push, hitFound flag out.
void orc_trace_ref_bvh2(const rq_bvh2_node* nodes, const rq_triangle* tris, const rq_ray* rays, uint32_t n,
                        float t_eps, uint32_t* flags_out, int threads) {
    parallel_for(n, threads, [&](uint32_t idx) {
        const rq_ray& r = rays[idx];
        V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
        auto clampd = [](float x) { return std::fabs(x) > 1e-8f ? x : (x >= 0.0f ? 1e-8f : -1e-8f); };
        V3 inv{1.0f / clampd(d.x), 1.0f / clampd(d.y), 1.0f / clampd(d.z)};
        float closestT = r.tmax;
        uint32_t hitFound = 0;
        auto box = [&](const rq_bvh2_node& nd, float& tb) {
            float t0x = (nd.aabb_min[0] - o.x) * inv.x, t1x = (nd.aabb_max[0] - o.x) * inv.x;
            float t0y = (nd.aabb_min[1] - o.y) * inv.y, t1y = (nd.aabb_max[1] - o.y) * inv.y;
            float t0z = (nd.aabb_min[2] - o.z) * inv.z, t1z = (nd.aabb_max[2] - o.z) * inv.z;
            float tNear = fmax_(fmax_(fmin_(t0x, t1x), fmin_(t0y, t1y)), fmin_(t0z, t1z));
            float tFar = fmin_(fmin_(fmax_(t0x, t1x), fmax_(t0y, t1y)), fmax_(t0z, t1z));
            tb = tNear;
            return (tFar >= fmax_(0.0f, tNear)) && (tNear < closestT);
        };
        uint32_t stack[32];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const rq_bvh2_node& nd = nodes[stack[--sp]];
            float tb;
            if (!box(nd, tb)) continue;
            if (nd.left_child < 0) {
                uint32_t start = uint32_t(~nd.left_child);
                for (int32_t i = 0; i < nd.right_child; ++i) {
                    const rq_triangle& tr = tris[start + uint32_t(i)];
                    V3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]},
                        v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                    float t, u, v;
                    if (!mt_test(o, d, v0, v1, v2, 1e-8f, t, u, v)) continue;
                    if (t > t_eps && t < closestT) {
                        closestT = t;
                        hitFound = 1;
                    }
                }
            } else {
                uint32_t l = uint32_t(nd.left_child), rr = uint32_t(nd.right_child);
                float tl, tr;
                bool hl = box(nodes[l], tl), hr = box(nodes[rr], tr);
                if (hl && hr) {
                    if (tl < tr) {
                        if (sp < 32) stack[sp++] = rr;
                        if (sp < 32) stack[sp++] = l;
                    } else {
                        if (sp < 32) stack[sp++] = l;
                        if (sp < 32) stack[sp++] = rr;
                    }
                } else if (hl) {
                    if (sp < 32) stack[sp++] = l;
                } else if (hr) {
                    if (sp < 32) stack[sp++] = rr;
                }
            }
        }
        flags_out[idx] = hitFound;
    });
}

// The engine's 4-wide traversal specification (see trace_bvh4 above).
// perm (may be NULL) maps leaf order to original IDs.  bary: 2 floats/ray.
void orc_trace_bvh4(const rq_bvh4_node* nodes, const rq_triangle* tris, const uint32_t* perm, const rq_ray* rays,
                    uint32_t n, uint32_t flags, rq_hit* hits, float* bary, rq_ray_stats* stats, int threads) {
    parallel_for(n, threads, [&](uint32_t i) {
        TraceOut t = trace_bvh4(nodes, tris, rays[i], flags);
        if (hits) {
            if (t.hit)
                hits[i] = {1u, t.t, 0u, perm ? perm[t.prim] : t.prim};
            else
                hits[i] = {0u, -1.0f, 0xffffffffu, 0xffffffffu};
        }
        if (bary) {
            bary[2 * size_t(i)] = t.hit ? t.u : 0.0f;
            bary[2 * size_t(i) + 1] = t.hit ? t.v : 0.0f;
        }
        if (stats) stats[i] = {t.hit ? 1u : 0u, t.boxes, t.tris, 0u};
    });
}

void orc_trace_radv(const uint8_t* img, const rq_ray* rays, uint32_t n, uint32_t flags, rq_hit* hits, float* bary,
                    int threads) {
    parallel_for(n, threads, [&](uint32_t i) {
        TraceOut t = trace_radv(img, rays[i], flags);
        if (hits) {
            if (t.hit)
                hits[i] = {1u, t.t, 0u, t.prim};
            else
                hits[i] = {0u, -1.0f, 0xffffffffu, 0xffffffffu};
        }
        if (bary) {
            bary[2 * size_t(i)] = t.hit ? t.u : 0.0f;
            bary[2 * size_t(i) + 1] = t.hit ? t.v : 0.0f;
        }
    });
}

// software_bvh_bvh4.comp:60-94 procedural rays, tmin 0.01 / tmax 1000.
void orc_gen_rays_procedural(const float cam[3], const float look[3], uint32_t count, uint32_t coherent,
                             rq_ray* rays) {
    V3 cp{cam[0], cam[1], cam[2]}, la{look[0], look[1], look[2]};
    V3 fwd = normalize(sub(la, cp));
    V3 right = normalize(cross(fwd, V3{0.0f, 1.0f, 0.0f}));
    V3 up = cross(right, fwd);
    for (uint32_t idx = 0; idx < count; ++idx) {
        V3 o, d;
        if (coherent) {
            uint32_t width = 1024, height = (count + width - 1) / width;
            uint32_t x = idx % width, y = idx / width;
            float u = ((float(x) + 0.5f) / float(width)) * 2.0f - 1.0f;
            float v = ((float(y) + 0.5f) / float(height)) * 2.0f - 1.0f;
            o = cp;
            d = normalize(add(add(fwd, mul(mul(right, u), 0.55f)), mul(mul(up, v), 0.55f)));
        } else {
            float rx = hash_float(idx * 6 + 0) * 80.0f - 40.0f;
            float ry = hash_float(idx * 6 + 1) * 15.0f + 15.0f;
            float rz = hash_float(idx * 6 + 2) * 80.0f - 40.0f;
            o = {rx, ry, rz};
            float dx = hash_float(idx * 6 + 3) * 0.8f - 0.4f;
            float dy = -1.0f - hash_float(idx * 6 + 4) * 0.5f;
            float dz = hash_float(idx * 6 + 5) * 0.8f - 0.4f;
            d = normalize(V3{dx, dy, dz});
        }
        rays[idx] = {{o.x, o.y, o.z}, 0.01f, {d.x, d.y, d.z}, 1000.0f};
    }
}

void orc_sincos(float x, float* s, float* c) { sincos_taylor(x, s, c); }

// Two-level scenes (rq_tlas_build + rq_tlas_trace).  Instance i uses BLAS
// blas_of[i] (arrays nodes4[b], tris[b], perm[b]) with the row-major 3x4
// object-to-world transform xf + 12i.  The top level is rebuilt here the way
// the engine builds it: inverse transforms in double (adjugate / det,
// translation -A^-1 t, rounded once), each instance's BLAS root box
// transformed corner by corner and widened by 2^-20 of the coordinate
// magnitudes, stored as the degenerate triangle (min, max, min), then the
// LBVH of those triangles with one per leaf.  Traversal: one stack; at an
// instance leaf the ray moves to object space (direction not renormalised),
// a marker entry and the BLAS root are pushed; popping the marker returns.
void orc_tlas_trace(const uint64_t* blas_nodes4, const uint64_t* blas_tris, const uint64_t* blas_perm,
                    const uint32_t* blas_of, const float* xf, const uint32_t* ids, const uint32_t* masks,
                    uint32_t ninst, const rq_ray* rays, uint32_t n, uint32_t flags, uint32_t cull, rq_hit* hits,
                    int threads) {
    std::vector<float> inv(12ull * ninst), tri9(9ull * ninst);
    for (uint32_t i = 0; i < ninst; ++i) {
        const float* f = xf + 12ull * i;
        const double a[3][3] = {{f[0], f[1], f[2]}, {f[4], f[5], f[6]}, {f[8], f[9], f[10]}};
        const double t[3] = {f[3], f[7], f[11]};
        const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
        const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
        const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
        const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
        double m[3][3];
        m[0][0] = c00 / det;
        m[0][1] = (a[0][2] * a[2][1] - a[0][1] * a[2][2]) / det;
        m[0][2] = (a[0][1] * a[1][2] - a[0][2] * a[1][1]) / det;
        m[1][0] = c01 / det;
        m[1][1] = (a[0][0] * a[2][2] - a[0][2] * a[2][0]) / det;
        m[1][2] = (a[0][2] * a[1][0] - a[0][0] * a[1][2]) / det;
        m[2][0] = c02 / det;
        m[2][1] = (a[0][1] * a[2][0] - a[0][0] * a[2][1]) / det;
        m[2][2] = (a[0][0] * a[1][1] - a[0][1] * a[1][0]) / det;
        for (int r = 0; r < 3; ++r) {
            const double tr = -((m[r][0] * t[0] + m[r][1] * t[1]) + m[r][2] * t[2]);
            for (int c = 0; c < 3; ++c) inv[12ull * i + 4 * r + c] = float(m[r][c]);
            inv[12ull * i + 4 * r + 3] = float(tr);
        }
        const rq_bvh4_node& root = reinterpret_cast<const rq_bvh4_node*>(blas_nodes4[blas_of[i]])[0];
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int k = 0; k < 4; ++k) {
            if (root.child_count[k] == 0) continue;
            lo[0] = fmin_(lo[0], root.min_x[k]);
            lo[1] = fmin_(lo[1], root.min_y[k]);
            lo[2] = fmin_(lo[2], root.min_z[k]);
            hi[0] = fmax_(hi[0], root.max_x[k]);
            hi[1] = fmax_(hi[1], root.max_y[k]);
            hi[2] = fmax_(hi[2], root.max_z[k]);
        }
        float wlo[3] = {INFINITY, INFINITY, INFINITY}, whi[3] = {-INFINITY, -INFINITY, -INFINITY};
        for (int c = 0; c < 8; ++c) {
            const float x = (c & 1) ? hi[0] : lo[0], y = (c & 2) ? hi[1] : lo[1], z = (c & 4) ? hi[2] : lo[2];
            for (int r = 0; r < 3; ++r) {
                const float w = ((f[4 * r] * x + f[4 * r + 1] * y) + f[4 * r + 2] * z) + f[4 * r + 3];
                wlo[r] = fmin_(wlo[r], w);
                whi[r] = fmax_(whi[r], w);
            }
        }
        for (int r = 0; r < 3; ++r) {
            const float pad = (std::fabs(wlo[r]) + std::fabs(whi[r])) * 0x1p-20f;
            tri9[9ull * i + r] = wlo[r] - pad;
            tri9[9ull * i + 3 + r] = whi[r] + pad;
            tri9[9ull * i + 6 + r] = wlo[r] - pad;
        }
    }
    std::vector<uint32_t> top_perm(ninst);
    std::vector<rq_bvh4_node> top4(ninst);
    std::vector<rq_bvh2_node> top2(2ull * ninst);
    uint32_t n2 = 0, n4 = 0, d4 = 0;
    orc_lbvh_build(tri9.data(), 3, nullptr, ninst, 1, nullptr, top_perm.data(), top2.data(), &n2, nullptr,
                   top4.data(), &n4, &d4);
    const bool any = flags & 1u, mt = flags & 2u;
    const int32_t kMarker = 0x40000000;
    parallel_for(n, threads, [&](uint32_t id) {
        const rq_ray& r = rays[id];
        const V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
        const float tmin = r.tmin;
        float best = r.tmax;
        auto setup = [](V3 oo, V3 dd, float* iv, float* oi) {
            iv[0] = safe_inv(dd.x);
            iv[1] = safe_inv(dd.y);
            iv[2] = safe_inv(dd.z);
            oi[0] = oo.x * iv[0];
            oi[1] = oo.y * iv[1];
            oi[2] = oo.z * iv[2];
        };
        float wi[3], wo[3], ci[3], co[3];
        setup(o, d, wi, wo);
        std::memcpy(ci, wi, sizeof(ci));
        std::memcpy(co, wo, sizeof(co));
        V3 oo = o, od = d;
        WtRay w = wt_setup(d);
        bool inside = false, hit = false;
        const rq_bvh4_node* nodes = top4.data();
        const rq_triangle* tris = nullptr;
        const uint32_t* perm = nullptr;
        uint32_t cur_id = 0, hit_inst = 0xffffffffu, hit_prim = 0xffffffffu;
        FixedStack<int32_t> st;
        st.push_back(0);
        bool done = false;
        while (!st.empty() && !done) {
            const int32_t e = st.back();
            st.pop_back();
            if (e == kMarker) {
                inside = false;
                nodes = top4.data();
                std::memcpy(ci, wi, sizeof(ci));
                std::memcpy(co, wo, sizeof(co));
                continue;
            }
            if (e >= 0) {
                const rq_bvh4_node& nd = nodes[e];
                int32_t he[4];
                float ht[4];
                int nh = 0;
                for (int k = 0; k < 4; ++k) {
                    if (nd.child_count[k] == 0) continue;
                    float tn;
                    if (slab4(ci, co, tmin, best, nd, k, tn)) {
                        const int32_t ent = nd.child_count[k] < 0
                                                ? nd.child_index[k]
                                                : int32_t(0x80000000u | (uint32_t(nd.child_count[k] - 1) << 27) |
                                                          uint32_t(~nd.child_index[k]));
                        int pos = nh;
                        if (!any)
                            while (pos > 0 && ht[pos - 1] > tn) {
                                he[pos] = he[pos - 1];
                                ht[pos] = ht[pos - 1];
                                --pos;
                            }
                        he[pos] = ent;
                        ht[pos] = tn;
                        ++nh;
                    }
                }
                for (int j = nh - 1; j >= 0; --j) st.push_back(he[j]);
                continue;
            }
            const uint32_t first = uint32_t(e) & 0x07ffffffu, cnt = ((uint32_t(e) >> 27) & 15u) + 1u;
            if (!inside) {
                const uint32_t i = top_perm[first];
                if ((masks[i] & cull) == 0u) continue;
                const float* m = inv.data() + 12ull * i;
                oo = V3{((m[0] * o.x + m[1] * o.y) + m[2] * o.z) + m[3], ((m[4] * o.x + m[5] * o.y) + m[6] * o.z) + m[7],
                        ((m[8] * o.x + m[9] * o.y) + m[10] * o.z) + m[11]};
                od = V3{(m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
                        (m[8] * d.x + m[9] * d.y) + m[10] * d.z};
                setup(oo, od, ci, co);
                w = wt_setup(od);
                const uint32_t b = blas_of[i];
                nodes = reinterpret_cast<const rq_bvh4_node*>(blas_nodes4[b]);
                tris = reinterpret_cast<const rq_triangle*>(blas_tris[b]);
                perm = reinterpret_cast<const uint32_t*>(blas_perm[b]);
                cur_id = ids[i];
                inside = true;
                st.push_back(kMarker);
                st.push_back(0);
                continue;
            }
            for (uint32_t p = first; p < first + cnt; ++p) {
                const rq_triangle& tr = tris[p];
                V3 v0{tr.v0[0], tr.v0[1], tr.v0[2]}, v1{tr.v1[0], tr.v1[1], tr.v1[2]}, v2{tr.v2[0], tr.v2[1], tr.v2[2]};
                float t, u, v;
                const bool ok = mt ? mt_test(oo, od, v0, v1, v2, 1e-7f, t, u, v) : wt_test(w, oo, v0, v1, v2, t, u, v);
                if (ok && t >= tmin && t < best) {
                    best = t;
                    hit = true;
                    hit_inst = cur_id;
                    hit_prim = perm[p];
                    if (any) {
                        done = true;
                        break;
                    }
                }
            }
        }
        rq_hit h;
        h.hit = hit ? 1u : 0u;
        h.t = hit ? best : -1.0f;
        h.instance_id = hit ? hit_inst : 0xffffffffu;
        h.primitive_id = hit ? hit_prim : 0xffffffffu;
        hits[id] = h;
    });
}

// Depth z/w of G-buffer positions under the column-major view-projection
// `vp` (1.0 where the pixel saw no geometry).
void orc_gbuffer_depth(const rq_gbuffer_px* g, uint32_t npix, const float* vp, float* depth) {
    for (uint32_t p = 0; p < npix; ++p) {
        if (g[p].vis == 0u) {
            depth[p] = 1.0f;
            continue;
        }
        const float x = g[p].pos[0], y = g[p].pos[1], z = g[p].pos[2];
        const float zc = ((vp[2] * x + vp[6] * y) + vp[10] * z) + vp[14];
        const float wc = ((vp[3] * x + vp[7] * y) + vp[11] * z) + vp[15];
        depth[p] = zc / wc;
    }
}

// One pass of shaders/bilateral_blur.comp:15-55 along (dx, dy): the 9-tap
// Gaussian with depth rejection, taps at whole texels clamped to the edge.
void orc_blur_ao(const float* in, const float* depth, float* out, uint32_t w, uint32_t h, int dx, int dy,
                 float threshold) {
    const float wt[4] = {0.1945946f, 0.1216216f, 0.054054f, 0.016216f};
    auto clampi = [](int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); };
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            const uint32_t p = y * w + x;
            const float cv = in[p], cd = depth[p];
            if (cd >= 1.0f) {
                out[p] = cv;
                continue;
            }
            float total = 0.227027f;
            float result = cv * total;
            for (int i = 1; i <= 4; ++i) {
                const uint32_t qp = uint32_t(clampi(int(y) + dy * i, 0, int(h) - 1)) * w +
                                    uint32_t(clampi(int(x) + dx * i, 0, int(w) - 1));
                const uint32_t qn = uint32_t(clampi(int(y) - dy * i, 0, int(h) - 1)) * w +
                                    uint32_t(clampi(int(x) - dx * i, 0, int(w) - 1));
                const float wp = wt[i - 1] * (std::fabs(depth[qp] - cd) < threshold ? 1.0f : 0.0f);
                result = result + in[qp] * wp;
                total = total + wp;
                const float wn = wt[i - 1] * (std::fabs(depth[qn] - cd) < threshold ? 1.0f : 0.0f);
                result = result + in[qn] * wn;
                total = total + wn;
            }
            out[p] = result / fmax_(total, 0.001f);
        }
}

// The generated rays of the serving requests (kind 1 shadow, 2 AO, 3
// closest), ray i from draws pcg_hash(base + k) / 2^32 with
// base = pcg_hash(seed ^ pcg_hash(i)).  Shadow and AO rays start on a point
// of triangle pcg_hash(base + 7) % ntri (folded barycentrics, face normal
// turned to +z): shadow toward a light in [-1,1]^2 x [2,2.5] from P + 0.04 N
// over [0.01, dist - 0.04] (shaders/tiled_lighting_ra.comp:118-148); AO a
// cosine-hemisphere direction from P + 0.03 N over [0.01, 0.5]
// (shaders/rq_ao.comp:32-45, 77-86).  any[i] = 1 for any-hit rays.
void orc_gen_mesh_rays(const float* pos, const uint32_t* idx, uint32_t ntri, uint32_t kind, uint32_t seed,
                       uint32_t n, rq_ray* rays, uint32_t* any) {
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t base = pcg_hash(seed ^ pcg_hash(i));
        auto draw = [&](uint32_t k) { return float(pcg_hash(base + k)) * kInv2Pow32; };
        V3 o, d;
        float tmin = 0.01f, tmax;
        if (kind == 3u) {
            o = {-1.0f + 2.0f * draw(0), -1.0f + 2.0f * draw(1), 2.0f};
            d = normalize(V3{-0.3f + 0.6f * draw(2), -0.3f + 0.6f * draw(3), -1.0f});
            tmax = 1000.0f;
        } else {
            const uint32_t t = pcg_hash(base + 7u) % ntri;
            auto vtx = [&](uint32_t v) { return V3{pos[3ull * v], pos[3ull * v + 1], pos[3ull * v + 2]}; };
            const V3 v0 = vtx(idx[3ull * t]), v1 = vtx(idx[3ull * t + 1]), v2 = vtx(idx[3ull * t + 2]);
            float a = draw(0), b = draw(1);
            if (a + b > 1.0f) {
                a = 1.0f - a;
                b = 1.0f - b;
            }
            const V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
            const V3 P{v0.x + (e1.x * a + e2.x * b), v0.y + (e1.y * a + e2.y * b), v0.z + (e1.z * a + e2.z * b)};
            V3 N = normalize(cross(e1, e2));
            if (N.z < 0.0f) N = {-N.x, -N.y, -N.z};
            if (kind == 1u) {
                const V3 L{-1.0f + 2.0f * draw(2), -1.0f + 2.0f * draw(3), 2.0f + 0.5f * draw(4)};
                const V3 tl = sub(L, P);
                const float dist = std::sqrt(dot(tl, tl));
                d = {tl.x / dist, tl.y / dist, tl.z / dist};
                o = {P.x + N.x * 0.04f, P.y + N.y * 0.04f, P.z + N.z * 0.04f};
                tmax = dist - 0.04f;
            } else {
                const float u1 = draw(2), u2 = draw(3);
                const float rr = std::sqrt(u1);
                const float theta = 6.2831853f * u2;
                float sn, cs;
                sincos_taylor(theta, &sn, &cs);
                const float x = rr * cs, y = rr * sn, z = std::sqrt(fmax_(0.0f, 1.0f - u1));
                const V3 up = std::fabs(N.z) < 0.999f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f};
                const V3 tg = normalize(cross(up, N));
                const V3 bt = cross(N, tg);
                d = normalize(V3{(tg.x * x + bt.x * y) + N.x * z, (tg.y * x + bt.y * y) + N.y * z,
                                 (tg.z * x + bt.z * y) + N.z * z});
                o = {P.x + N.x * 0.03f, P.y + N.y * 0.03f, P.z + N.z * 0.03f};
                tmax = 0.5f;
            }
        }
        rays[i] = rq_ray{{o.x, o.y, o.z}, tmin, {d.x, d.y, d.z}, tmax};
        if (any) any[i] = kind == 3u ? 0u : 1u;
    }
}

}  // extern "C"

namespace {

// Primary ray of visbuf_raycast.comp:15-51 for one pixel (optional per-pixel
// jitter from the camera's seed).
rq_ray camera_ray(const rq_camera& c, uint32_t pixel) {
    const uint32_t px = pixel % c.width, py = pixel / c.width;
    float jx = 0.5f, jy = 0.5f;
    if (c.jitter) {
        uint32_t h = pcg_hash(c.seed ^ pcg_hash(pixel));
        jx = float(h) * kInv2Pow32;
        jy = float(pcg_hash(h)) * kInv2Pow32;
    }
    const float u = (float(px) + jx) / float(c.width);
    const float v = (float(py) + jy) / float(c.height);
    const float cl[4] = {u * 2.0f - 1.0f, v * 2.0f - 1.0f, 1.0f, 1.0f};
    float wt[4];
    mat4_mul(c.inv_view_proj, cl, wt);
    const V3 o{c.cam_pos[0], c.cam_pos[1], c.cam_pos[2]};
    const V3 target{wt[0] / wt[3], wt[1] / wt[3], wt[2] / wt[3]};
    const V3 d = normalize(sub(target, o));
    return rq_ray{{o.x, o.y, o.z}, c.tmin, {d.x, d.y, d.z}, c.tmax};
}

// hemisphereSample of rq_ao.comp:32-45: two draws of the one-at-a-time hash
// advance `seed`; sin/cos through sincos_taylor.
V3 hemisphere_dir(V3 N, uint32_t& seed) {
    seed = ao_hash(seed);
    const float u1 = float(seed) * kInv2Pow32;
    seed = ao_hash(seed);
    const float u2 = float(seed) * kInv2Pow32;
    const float rr = std::sqrt(u1);
    const float theta = 6.2831853f * u2;
    float sn, cs;
    sincos_taylor(theta, &sn, &cs);
    const float x = rr * cs, y = rr * sn, z = std::sqrt(fmax_(0.0f, 1.0f - u1));
    const V3 up = std::fabs(N.z) < 0.999f ? V3{0.0f, 0.0f, 1.0f} : V3{1.0f, 0.0f, 0.0f};
    const V3 tg = normalize(cross(up, N));
    const V3 bt = cross(N, tg);
    return normalize(V3{(tg.x * x + bt.x * y) + N.x * z, (tg.y * x + bt.y * y) + N.y * z,
                        (tg.z * x + bt.z * y) + N.z * z});
}

// The secondary rays of one G-buffer pixel, in the order the frame casts
// them: emit(slot, ray) for every light k that casts a shadow ray
// (shaders/tiled_lighting_ra.comp:118-148; slot k) and every AO sample s
// (shaders/rq_ao.comp:70-94 with the G-buffer's position and normal; slot
// 32 + s).  Pixels without geometry cast nothing.
template <class F>
void shade_pixel_rays(const rq_gbuffer_px& g, const rq_shade_params& p, uint32_t pixel, F&& emit) {
    if (g.vis == 0u) return;
    const V3 P{g.pos[0], g.pos[1], g.pos[2]}, N{g.nrm[0], g.nrm[1], g.nrm[2]};
    const V3 os{P.x + N.x * p.shadow_bias, P.y + N.y * p.shadow_bias, P.z + N.z * p.shadow_bias};
    for (uint32_t k = 0; k < p.num_lights; ++k) {
        const rq_light& L0 = p.lights[k];
        const V3 tl{L0.pos[0] - P.x, L0.pos[1] - P.y, L0.pos[2] - P.z};
        const float dist = std::sqrt(dot(tl, tl));
        if (dist > L0.radius || dist < 0.001f) continue;
        const V3 L{tl.x / dist, tl.y / dist, tl.z / dist};
        if (fmax_(0.0f, dot(N, L)) <= 0.0f) continue;
        emit(k, rq_ray{{os.x, os.y, os.z}, p.shadow_tmin, {L.x, L.y, L.z}, dist - p.shadow_bias});
    }
    if (p.ao_spp) {
        uint32_t seed = pixel + 5544u;
        const V3 oa{P.x + N.x * p.ao_bias, P.y + N.y * p.ao_bias, P.z + N.z * p.ao_bias};
        for (uint32_t s = 0; s < p.ao_spp; ++s) {
            const V3 dir = hemisphere_dir(N, seed);
            emit(32u + s, rq_ray{{oa.x, oa.y, oa.z}, p.ao_tmin, {dir.x, dir.y, dir.z}, p.ao_tmax});
        }
    }
}

// The reflection ray of shaders/tiled_lighting_ra.comp:91-113 for one
// G-buffer pixel: R = reflect(normalize(P - cam), N) (GLSL reflect:
// I - 2 dot(N, I) N), from P + bias N over [tmin, tmax].
rq_ray reflect_ray(const rq_gbuffer_px& g, const rq_reflect_params& p) {
    const V3 P{g.pos[0], g.pos[1], g.pos[2]}, N{g.nrm[0], g.nrm[1], g.nrm[2]};
    const V3 V = normalize(sub(P, V3{p.cam_pos[0], p.cam_pos[1], p.cam_pos[2]}));
    const float k = 2.0f * dot(N, V);
    const V3 R{V.x - k * N.x, V.y - k * N.y, V.z - k * N.z};
    return rq_ray{{P.x + N.x * p.bias, P.y + N.y * p.bias, P.z + N.z * p.bias}, p.tmin, {R.x, R.y, R.z}, p.tmax};
}

// rq_ao.comp:47-69 for one pixel: the world position reconstructed from the
// depth at the pixel centre through inv_view_proj, the normal from the
// cross product of the right and upper neighbours' reconstructed positions
// (depth read clamped at the image edge, as a clamp-to-edge sampler at texel
// centres reads it), turned toward the camera.  Returns false where
// depth >= 1 (no geometry).
bool ao_depth_surface(const float* depth, const rq_ao_depth_params& p, uint32_t px, uint32_t py, V3& P, V3& N) {
    const uint32_t w = p.width, h = p.height;
    const float d = depth[size_t(py) * w + px];
    if (d >= 1.0f) return false;
    const float fw = float(w), fh = float(h);
    const float u = (float(px) + 0.5f) / fw, v = (float(py) + 0.5f) / fh;
    const float tx = 1.0f / fw, ty = 1.0f / fh;
    const float dr = depth[size_t(py) * w + (px + 1 < w ? px + 1 : w - 1)];
    const float du = depth[size_t(py + 1 < h ? py + 1 : h - 1) * w + px];
    auto unproject = [&](float uu, float vv, float dd) {
        const float ndc[4] = {uu * 2.0f - 1.0f, vv * 2.0f - 1.0f, dd, 1.0f};
        float o[4];
        mat4_mul(p.inv_view_proj, ndc, o);
        return V3{o[0] / o[3], o[1] / o[3], o[2] / o[3]};
    };
    P = unproject(u, v, d);
    const V3 pr = unproject(u + tx, v, dr);
    const V3 pu = unproject(u, v + ty, du);
    N = normalize(cross(sub(pr, P), sub(pu, P)));
    if (dot(N, sub(V3{p.cam_pos[0], p.cam_pos[1], p.cam_pos[2]}, P)) < 0.0f) N = {-N.x, -N.y, -N.z};
    return true;
}

// The AO rays of one pixel of rq_ao.comp:70-94 from a reconstructed surface:
// max(1, spp) samples seeded y*W + x + 5544, from P + bias N.
template <class F>
void ao_depth_rays(const rq_ao_depth_params& p, uint32_t pixel, V3 P, V3 N, F&& emit) {
    uint32_t seed = pixel + 5544u;
    const uint32_t spp = p.spp > 1u ? p.spp : 1u;
    const V3 o{P.x + N.x * p.bias, P.y + N.y * p.bias, P.z + N.z * p.bias};
    for (uint32_t s = 0; s < spp; ++s) {
        const V3 dir = hemisphere_dir(N, seed);
        emit(s, rq_ray{{o.x, o.y, o.z}, p.tmin, {dir.x, dir.y, dir.z}, p.max_distance});
    }
}

// Box of one triangle (as the builds compute it) and unions.
struct Box {
    float mn[3], mx[3];
};
inline Box tri_box(const rq_triangle& t) {
    Box b;
    for (int a = 0; a < 3; ++a) {
        b.mn[a] = fmin_(fmin_(t.v0[a], t.v1[a]), t.v2[a]);
        b.mx[a] = fmax_(fmax_(t.v0[a], t.v1[a]), t.v2[a]);
    }
    return b;
}
inline Box box_union(const Box& a, const Box& b) {
    Box r;
    for (int k = 0; k < 3; ++k) {
        r.mn[k] = fmin_(a.mn[k], b.mn[k]);
        r.mx[k] = fmax_(a.mx[k], b.mx[k]);
    }
    return r;
}
Box range_box(const rq_triangle* tris, uint32_t first, uint32_t count) {
    Box b = tri_box(tris[first]);
    for (uint32_t i = 1; i < count; ++i) b = box_union(b, tri_box(tris[first + i]));
    return b;
}

Box refit2(rq_bvh2_node* n, const rq_triangle* tris, int32_t i) {
    rq_bvh2_node& nd = n[i];
    Box b;
    if (nd.left_child < 0)
        b = range_box(tris, uint32_t(~nd.left_child), uint32_t(nd.right_child));
    else
        b = box_union(refit2(n, tris, nd.left_child), refit2(n, tris, nd.right_child));
    for (int a = 0; a < 3; ++a) {
        nd.aabb_min[a] = b.mn[a];
        nd.aabb_max[a] = b.mx[a];
    }
    return b;
}

Box refit4(rq_bvh4_node* n, const rq_triangle* tris, int32_t i) {
    rq_bvh4_node& nd = n[i];
    Box all{{INFINITY, INFINITY, INFINITY}, {-INFINITY, -INFINITY, -INFINITY}};
    for (int k = 0; k < 4; ++k) {
        if (nd.child_count[k] == 0) continue;
        const Box b = nd.child_count[k] < 0 ? refit4(n, tris, nd.child_index[k])
                                            : range_box(tris, uint32_t(~nd.child_index[k]), uint32_t(nd.child_count[k]));
        nd.min_x[k] = b.mn[0];
        nd.min_y[k] = b.mn[1];
        nd.min_z[k] = b.mn[2];
        nd.max_x[k] = b.mx[0];
        nd.max_y[k] = b.mx[1];
        nd.max_z[k] = b.mx[2];
        all = box_union(all, b);
    }
    return all;
}

// SplitMix64 with a (0, 1] double draw: the workload generator's PRNG.
struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return double((next() >> 11) + 1) * (1.0 / 9007199254740992.0); }
};

}  // namespace

extern "C" {

// Primary rays of visbuf_raycast.comp:15-51 (optional per-pixel jitter),
// closest hit with the engine traversal, G-buffer pixel as rq_render_gbuffer
// writes it.  `pixels` lists the pixel indices to evaluate (NULL = all);
// out[i] receives pixel pixels[i].
void orc_render_gbuffer(const rq_bvh4_node* nodes, const rq_triangle* tris, const uint32_t* perm, const rq_camera* cam,
                        const uint32_t* pixels, uint32_t npix, rq_gbuffer_px* out, int threads) {
    const rq_camera c = *cam;
    parallel_for(npix, threads, [&](uint32_t i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        const rq_ray r = camera_ray(c, pixel);
        const V3 o{r.org[0], r.org[1], r.org[2]}, d{r.dir[0], r.dir[1], r.dir[2]};
        TraceOut t = trace_bvh4(nodes, tris, r, c.flags & 2u);
        rq_gbuffer_px g;
        if (!t.hit) {
            g = {{0.0f, 0.0f, 0.0f}, 0u, {0.0f, 0.0f, 0.0f}, -1.0f};
        } else {
            V3 p{o.x + t.t * d.x, o.y + t.t * d.y, o.z + t.t * d.z};
            const rq_triangle& tr = tris[t.prim];
            V3 e1{tr.v1[0] - tr.v0[0], tr.v1[1] - tr.v0[1], tr.v1[2] - tr.v0[2]};
            V3 e2{tr.v2[0] - tr.v0[0], tr.v2[1] - tr.v0[1], tr.v2[2] - tr.v0[2]};
            V3 n = normalize(cross(e1, e2));
            if (dot(n, sub(o, p)) < 0.0f) n = {-n.x, -n.y, -n.z};
            uint32_t pid = perm ? perm[t.prim] : t.prim;
            g = {{p.x, p.y, p.z}, pid + 1u, {n.x, n.y, n.z}, t.t};
        }
        out[i] = g;
    });
}

// The primary rays themselves (rays[i] for pixel pixels[i], NULL = all).
void orc_camera_rays(const rq_camera* cam, const uint32_t* pixels, uint32_t npix, rq_ray* rays) {
    for (uint32_t i = 0; i < npix; ++i) rays[i] = camera_ray(*cam, pixels ? pixels[i] : i);
}

// Shadow rays of shaders/tiled_lighting_ra.comp:118-148 and AO rays of
// rq_ao.comp:18-94 for the listed pixels of a full-size G-buffer.
void orc_render_shadow_ao(const rq_bvh4_node* nodes, const rq_triangle* tris, const rq_gbuffer_px* gbuf,
                          const rq_shade_params* prm, const uint32_t* pixels, uint32_t npix, uint32_t* mask, float* ao,
                          uint64_t* rays_out, int threads) {
    const rq_shade_params p = *prm;
    std::atomic<uint64_t> total{0};
    parallel_for(npix, threads, [&](uint32_t i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        const rq_gbuffer_px& g = gbuf[pixel];
        uint32_t m = 0, rays = 0;
        float unocc = 0.0f;
        shade_pixel_rays(g, p, pixel, [&](uint32_t slot, const rq_ray& r) {
            ++rays;
            const bool hit = trace_bvh4(nodes, tris, r, 1u | (p.flags & 2u)).hit;
            if (hit) return;
            if (slot < 32u)
                m |= 1u << slot;
            else
                unocc += 1.0f;
        });
        mask[i] = m;
        ao[i] = (g.vis != 0u && p.ao_spp) ? unocc / float(p.ao_spp) : 1.0f;
        total += rays;
    });
    if (rays_out) *rays_out = total;
}

// The secondary rays of the listed pixels, in casting order: rays[j] with
// ray_pixel[j] = its index into `pixels` and ray_slot[j] = light k (< 32) or
// 32 + AO sample.  At most `cap` rays are written; *count gets the total.
void orc_shade_rays(const rq_gbuffer_px* gbuf, const rq_shade_params* prm, const uint32_t* pixels, uint32_t npix,
                    rq_ray* rays, uint32_t* ray_pixel, uint32_t* ray_slot, uint64_t cap, uint64_t* count) {
    const rq_shade_params p = *prm;
    uint64_t n = 0;
    for (uint32_t i = 0; i < npix; ++i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        shade_pixel_rays(gbuf[pixel], p, pixel, [&](uint32_t slot, const rq_ray& r) {
            if (n < cap) {
                rays[n] = r;
                ray_pixel[n] = i;
                ray_slot[n] = slot;
            }
            ++n;
        });
    }
    *count = n;
}

// Reflection closest-hit rays (shaders/tiled_lighting_ra.comp:91-113) for
// the listed pixels: hits[i] is rq_render_reflect's record of pixel
// pixels[i] (original primitive id; a miss record where the G-buffer pixel
// saw nothing).  rays (may be NULL) receives the rays themselves.
void orc_render_reflect(const rq_bvh4_node* nodes, const rq_triangle* tris, const uint32_t* perm,
                        const rq_gbuffer_px* gbuf, const rq_reflect_params* prm, const uint32_t* pixels,
                        uint32_t npix, rq_hit* hits, rq_ray* rays, int threads) {
    const rq_reflect_params p = *prm;
    parallel_for(npix, threads, [&](uint32_t i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        const rq_gbuffer_px& g = gbuf[pixel];
        if (g.vis == 0u) {
            hits[i] = {0u, -1.0f, 0xffffffffu, 0xffffffffu};
            if (rays) rays[i] = rq_ray{{0.0f, 0.0f, 0.0f}, 0.0f, {0.0f, 0.0f, 0.0f}, -1.0f};
            return;
        }
        const rq_ray r = reflect_ray(g, p);
        if (rays) rays[i] = r;
        const TraceOut t = trace_bvh4(nodes, tris, r, p.flags & 2u);
        hits[i] = t.hit ? rq_hit{1u, t.t, 0u, perm ? perm[t.prim] : t.prim}
                        : rq_hit{0u, -1.0f, 0xffffffffu, 0xffffffffu};
    });
}

// rq_ao.comp:47-97 from a depth buffer: ao[i] for pixel pixels[i] (NULL =
// all): 1.0 where depth >= 1, else the unoccluded fraction of max(1, spp)
// any-hit rays.  rays_out (may be NULL) accumulates the rays cast.
void orc_render_ao_depth(const rq_bvh4_node* nodes, const rq_triangle* tris, const float* depth,
                         const rq_ao_depth_params* prm, const uint32_t* pixels, uint32_t npix, float* ao,
                         uint64_t* rays_out, int threads) {
    const rq_ao_depth_params p = *prm;
    std::atomic<uint64_t> total{0};
    parallel_for(npix, threads, [&](uint32_t i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        V3 P, N;
        if (!ao_depth_surface(depth, p, pixel % p.width, pixel / p.width, P, N)) {
            ao[i] = 1.0f;
            return;
        }
        float unocc = 0.0f;
        uint32_t rays = 0;
        ao_depth_rays(p, pixel, P, N, [&](uint32_t, const rq_ray& r) {
            ++rays;
            if (!trace_bvh4(nodes, tris, r, 1u | (p.flags & 2u)).hit) unocc += 1.0f;
        });
        ao[i] = unocc / float(p.spp > 1u ? p.spp : 1u);
        total += rays;
    });
    if (rays_out) *rays_out = total;
}

// The AO rays of rq_ao.comp for the listed pixels, in order (ray_pixel[j]:
// index into `pixels`); pixels at depth >= 1 cast none.
void orc_ao_depth_rays(const float* depth, const rq_ao_depth_params* prm, const uint32_t* pixels, uint32_t npix,
                       rq_ray* rays, uint32_t* ray_pixel, uint64_t cap, uint64_t* count) {
    const rq_ao_depth_params p = *prm;
    uint64_t n = 0;
    for (uint32_t i = 0; i < npix; ++i) {
        const uint32_t pixel = pixels ? pixels[i] : i;
        V3 P, N;
        if (!ao_depth_surface(depth, p, pixel % p.width, pixel / p.width, P, N)) continue;
        ao_depth_rays(p, pixel, P, N, [&](uint32_t, const rq_ray& r) {
            if (n < cap) {
                rays[n] = r;
                ray_pixel[n] = i;
            }
            ++n;
        });
    }
    *count = n;
}

// Refit of a built tree to moved geometry: tris (leaf order, written) from
// pos/idx through perm, then every binary and 4-wide box as the union of
// the triangle boxes below it.  The topology (child links, counts) is kept.
void orc_refit(const float* pos, const uint32_t* idx, const uint32_t* perm, uint32_t n, rq_triangle* tris,
               rq_bvh2_node* nodes2, uint32_t n2, rq_bvh4_node* nodes4, uint32_t n4) {
    for (uint32_t i = 0; i < n; ++i) {
        V3 p0, p1, p2;
        tri_vertices(pos, 3, idx, perm[i], p0, p1, p2);
        tris[i] = rq_triangle{{p0.x, p0.y, p0.z, 0.0f}, {p1.x, p1.y, p1.z, 0.0f}, {p2.x, p2.y, p2.z, 0.0f}};
    }
    if (nodes2 && n2) refit2(nodes2, tris, 0);
    if (nodes4 && n4) refit4(nodes4, tris, 0);
}

// Leaf-order -> input triangle ids by the 9 float bit patterns of every
// triangle (the reference's SoftwareBVH drops its permutation,
// common/software_bvh.hpp:60-63).  Returns 0, or 1 when the input
// triangles are not unique by their bits or a leaf triangle is not found.
int orc_recover_perm(const rq_triangle* leaf_tris, uint32_t n, const float* pos, const uint32_t* idx, uint32_t ninput,
                     uint32_t* perm) {
    struct Key {
        uint32_t w[9];
    };
    auto key_of_input = [&](uint32_t t) {
        Key k;
        for (int c = 0; c < 3; ++c) std::memcpy(k.w + 3 * c, pos + 3ull * idx[3ull * t + c], 12);
        return k;
    };
    auto key_of_leaf = [&](uint32_t i) {
        Key k;
        std::memcpy(k.w, leaf_tris[i].v0, 12);
        std::memcpy(k.w + 3, leaf_tris[i].v1, 12);
        std::memcpy(k.w + 6, leaf_tris[i].v2, 12);
        return k;
    };
    auto less = [](const Key& a, const Key& b) { return std::memcmp(a.w, b.w, 36) < 0; };
    std::vector<std::pair<Key, uint32_t>> in(ninput);
    for (uint32_t t = 0; t < ninput; ++t) in[t] = {key_of_input(t), t};
    std::sort(in.begin(), in.end(), [&](const auto& a, const auto& b) { return less(a.first, b.first); });
    for (uint32_t t = 1; t < ninput; ++t)
        if (!less(in[t - 1].first, in[t].first)) return 1;
    for (uint32_t i = 0; i < n; ++i) {
        const Key k = key_of_leaf(i);
        auto it = std::lower_bound(in.begin(), in.end(), k, [&](const auto& a, const Key& b) { return less(a.first, b); });
        if (it == in.end() || std::memcmp(it->first.w, k.w, 36) != 0) return 1;
        perm[i] = it->second;
    }
    return 0;
}

// The benchmark workloads' height-field grid, restated from the engine's
// host generator so the reference arm of the benchmark can build its inputs
// without the engine: vertices on a (qx+1) x (qy+1) lattice over
// [x0,x1] x [y0,y1], z = amp sin(freq x) cos(freq y) + N(0, sigma) (SplitMix64
// draws through Box-Muller in double, rounded to float once); each quad
// (i, j) gives triangles (v00, v10, v01) and (v10, v11, v01), row-major.
int orc_scene_grid(uint32_t qx, uint32_t qy, float x0, float x1, float y0, float y1, float amp, float freq,
                   float sigma, uint64_t seed, float* pos, uint32_t* idx) {
    if (qx == 0 || qy == 0) return 1;
    const uint32_t nvx = qx + 1, nvy = qy + 1;
    if (pos) {
        SplitMix64 rng{seed};
        const double two_pi = 6.283185307179586476925286766559;
        double spare = 0.0;
        bool have_spare = false;
        for (uint32_t j = 0; j < nvy; ++j) {
            const double y = double(y0) + (double(y1) - double(y0)) * double(j) / double(qy);
            for (uint32_t i = 0; i < nvx; ++i) {
                const double x = double(x0) + (double(x1) - double(x0)) * double(i) / double(qx);
                double g;
                if (have_spare) {
                    g = spare;
                    have_spare = false;
                } else {
                    const double u1 = rng.uniform(), u2 = rng.uniform();
                    const double r = std::sqrt(-2.0 * std::log(u1));
                    g = r * std::cos(two_pi * u2);
                    spare = r * std::sin(two_pi * u2);
                    have_spare = true;
                }
                const double z = double(amp) * std::sin(double(freq) * x) * std::cos(double(freq) * y) +
                                 double(sigma) * g;
                float* p = pos + 3ull * (size_t(j) * nvx + i);
                p[0] = float(x);
                p[1] = float(y);
                p[2] = float(z);
            }
        }
    }
    if (idx) {
        uint32_t* o = idx;
        for (uint32_t j = 0; j < qy; ++j)
            for (uint32_t i = 0; i < qx; ++i) {
                const uint32_t v00 = j * nvx + i, v10 = v00 + 1, v01 = v00 + nvx, v11 = v01 + 1;
                o[0] = v00;
                o[1] = v10;
                o[2] = v01;
                o[3] = v10;
                o[4] = v11;
                o[5] = v01;
                o += 6;
            }
    }
    return 0;
}

// The benchmark camera (restated from the engine's host helper): right-handed
// look-at view and a Vulkan perspective (depth 0..1, y flipped, near 0.1,
// far 100), multiplied and inverted in double, stored column-major as float.
int orc_camera_look_at(const float eye[3], const float target[3], const float up[3], float fovy_deg, uint32_t width,
                       uint32_t height, rq_camera* out) {
    double e[3] = {eye[0], eye[1], eye[2]}, t[3] = {target[0], target[1], target[2]}, u0[3] = {up[0], up[1], up[2]};
    auto norm = [](double* v) {
        const double l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        v[0] /= l;
        v[1] /= l;
        v[2] /= l;
    };
    auto cross3 = [](const double* a, const double* b, double* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    double f[3] = {t[0] - e[0], t[1] - e[1], t[2] - e[2]};
    norm(f);
    double sx[3], ux[3];
    cross3(f, u0, sx);
    norm(sx);
    cross3(sx, f, ux);
    const double V[4][4] = {{sx[0], ux[0], -f[0], 0}, {sx[1], ux[1], -f[1], 0}, {sx[2], ux[2], -f[2], 0},
                            {-(sx[0] * e[0] + sx[1] * e[1] + sx[2] * e[2]),
                             -(ux[0] * e[0] + ux[1] * e[1] + ux[2] * e[2]), f[0] * e[0] + f[1] * e[1] + f[2] * e[2], 1}};
    const double aspect = double(width) / double(height);
    const double th = std::tan(double(fovy_deg) * 3.14159265358979323846 / 360.0);
    const double zn = 0.1, zf = 100.0;
    const double Pm[4][4] = {{1.0 / (aspect * th), 0, 0, 0},
                             {0, -1.0 / th, 0, 0},
                             {0, 0, zf / (zn - zf), -1},
                             {0, 0, -(zf * zn) / (zf - zn), 0}};
    double A[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            double acc = 0;
            for (int k = 0; k < 4; ++k) acc += Pm[k][r] * V[c][k];
            A[r][c] = acc;
            A[r][4 + c] = r == c ? 1.0 : 0.0;
        }
    for (int col = 0; col < 4; ++col) {
        int piv = col;
        for (int r = col + 1; r < 4; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
        if (std::fabs(A[piv][col]) < 1e-300) return 1;
        if (piv != col)
            for (int k = 0; k < 8; ++k) std::swap(A[piv][k], A[col][k]);
        const double d = A[col][col];
        for (int k = 0; k < 8; ++k) A[col][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != col) {
                const double m = A[r][col];
                for (int k = 0; k < 8; ++k) A[r][k] -= m * A[col][k];
            }
    }
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) out->inv_view_proj[4 * c + r] = float(A[r][4 + c]);
    out->cam_pos[0] = eye[0];
    out->cam_pos[1] = eye[1];
    out->cam_pos[2] = eye[2];
    out->width = width;
    out->height = height;
    out->jitter = 0;
    out->seed = 0;
    out->tmin = 0.01f;
    out->tmax = 10000.0f;
    out->flags = 0;
    return 0;
}

}  // extern "C"
