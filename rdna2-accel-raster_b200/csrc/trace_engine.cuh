// trace_engine.cuh — persistent traversal with per-lane ray refill.
//
// Every lane of a warp owns one ray at a time.  Ray ids come from a global
// counter in chunks of 32 (one atomic per chunk); whenever lanes are idle,
// a ballot and a rank within the idle mask hand them the next ids, so a warp
// keeps 32 rays in flight until the ids run out.  Each round:
//   1. inner phase — lanes without a pending leaf pop stack entries; an inner
//      node is box-tested and its hit children pushed (closest hit: sorted
//      near-to-far and pushed far-first; any hit: slot 3..0), a leaf entry is
//      parked as the lane's pending leaf; the phase ends when no lane wants
//      another inner node (every lane parked a leaf or ran out of entries);
//   2. leaf phase — lanes test their parked leaf's triangles in order;
//   3. lanes whose stack is empty, or whose any-hit ray found a hit, report
//      the result to the ray source and become idle.
// With INLOOP, lanes whose stack runs out during the inner phase report at
// once and idle lanes are refilled inside the inner phase too, which then
// ends only when no lane searches or `leaf_batch` lanes hold a parked leaf:
// rays that need few nodes no longer wait for the warp's longest one.
// Per ray this visits stack entries in exactly the order of a sequential
// pop-process-push traversal, so results do not depend on which lane or
// round a ray runs in and match the oracle's traversal bit for bit.  The
// stack's top entry is held in a register (the first child to visit after a
// node never goes through shared memory).
//
// A ray source provides:
//   uint32_t total;                                 number of ray ids
//   bool make(uint32_t id, Ray& r, Meta& m);        false = no ray for this id
//   void finish(uint32_t id, const Meta& m, const Ray& r, const Hit& h);
//   optional: kRoundEnd = true and void round_end(bool finished, const Meta& m).
#pragma once

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

constexpr int32_t kNoLeaf = 0;  // leaf entries always have bit 31 set
constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kChunk = 32;  // default ray ids per refill atomic

struct Ray {
    F3 o, d;
    float tmin, tmax;
    // set by sources that trace many BVHs in one launch (Src::kMulti)
    const rq_bvh4_node* nodes;
    const rq_triangle* tris;
    bool any;  // per-ray any hit (ANY == kAnyPerRay)
};

// ANY template argument: 0 closest hit, 1 any hit, kAnyPerRay = Ray::any.
constexpr int kAnyPerRay = 2;

template <class Src, class = void>
struct IsMulti {
    static constexpr bool value = false;
};
template <class Src>
struct IsMulti<Src, decltype(void(Src::kMulti))> {
    static constexpr bool value = Src::kMulti;
};

// Sources with kRoundEnd get round_end(finished, meta) once per round from
// all 32 lanes together (finished: this lane reported a ray this round;
// meta: that ray's), e.g. to count completions with one atomic per group.
template <class Src, class = void>
struct HasRoundEnd {
    static constexpr bool value = false;
};
template <class Src>
struct HasRoundEnd<Src, decltype(void(Src::kRoundEnd))> {
    static constexpr bool value = Src::kRoundEnd;
};

struct Hit {
    bool hit;
    float t;
    uint32_t idx;  // leaf-order primitive index
    float u, v;
    uint32_t boxes, tris;
};

// ----------------------------------------------------------- top levels
// The top TOP levels of a 4-wide tree (at most (4^TOP - 1) / 3 nodes, the
// root first, breadth-first) staged in shared memory by every block.  A
// staged node occupies kTopStride float4 (144 B: node k starts 4 banks
// after node k-1, so 16-B reads of different nodes by one quarter-warp do
// not collide); its inner children that are staged too have child index
// kStaged | slot.  Stack entries with kStaged name a shared-memory slot.
constexpr int32_t kStaged = 0x40000000;
constexpr int kTopStride = 9;

template <int TOP>
struct TopLevels {
    static constexpr int kMax = TOP <= 0 ? 0 : ((1 << (2 * TOP)) - 1) / 3;
    // shared memory: the nodes, slot -> global index, slot x child -> slot, count
    static constexpr size_t kBytes = TOP <= 0 ? 0 : size_t(kMax) * kTopStride * 16 + size_t(kMax) * 5 * 4 + 16;
};

// Stage the top levels (call with the whole block, before any traversal).
// `s_top` points at TopLevels<TOP>::kBytes of 16-B aligned shared memory.
template <int TOP>
__device__ __forceinline__ void stage_top(const rq_bvh4_node* __restrict__ nodes, float4* s_top) {
    constexpr int kMax = TopLevels<TOP>::kMax;
    int32_t* s_g = reinterpret_cast<int32_t*>(s_top + kMax * kTopStride);
    int32_t* s_c = s_g + kMax;
    uint32_t* s_n = reinterpret_cast<uint32_t*>(s_c + 4 * kMax);
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        for (int i = lane; i < 4 * kMax; i += 32) s_c[i] = -1;
        if (lane == 0) s_g[0] = 0;
        __syncwarp();
        uint32_t n = 1, lo = 0, hi = 1;
        for (int lvl = 1; lvl < TOP; ++lvl) {
            for (uint32_t b = lo; b < hi; b += 32) {
                const uint32_t s = b + lane;
                int4 ci = make_int4(0, 0, 0, 0), cc = make_int4(0, 0, 0, 0);
                if (s < hi) {
                    const int4* np = reinterpret_cast<const int4*>(nodes + s_g[s]);
                    ci = __ldg(np + 6);
                    cc = __ldg(np + 7);
                }
                const int32_t x[4] = {ci.x, ci.y, ci.z, ci.w}, c[4] = {cc.x, cc.y, cc.z, cc.w};
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const bool inner = s < hi && c[k] < 0;
                    const uint32_t m = __ballot_sync(kFull, inner);
                    if (inner) {
                        const uint32_t slot = n + __popc(m & ((1u << lane) - 1u));
                        s_g[slot] = x[k];
                        s_c[4 * s + k] = int32_t(slot);
                    }
                    n += __popc(m);
                }
                __syncwarp();
            }
            lo = hi;
            hi = n;
        }
        if (lane == 0) *s_n = n;
    }
    __syncthreads();
    const uint32_t n = *s_n;
    for (uint32_t i = threadIdx.x; i < n * 8u; i += blockDim.x) {
        const uint32_t s = i >> 3, j = i & 7u;
        float4 v = __ldg(reinterpret_cast<const float4*>(nodes + s_g[s]) + j);
        if (j == 6) {
            int32_t ci[4] = {__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z), __float_as_int(v.w)};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (s_c[4 * s + k] >= 0) ci[k] = kStaged | s_c[4 * s + k];
            v = make_float4(__int_as_float(ci[0]), __int_as_float(ci[1]), __int_as_float(ci[2]), __int_as_float(ci[3]));
        }
        s_top[s * kTopStride + j] = v;
    }
    __syncthreads();
}

// STACK bounds the entries per lane (stk has STACK rows of STRIDE words);
// stack_cap, if smaller, is the bound actually allocated.  CHUNK: ray ids
// taken per atomic.  refill_min: idle lanes get new rays only once at least
// this many lanes of the warp are idle (or all are), so that lanes join in
// groups and a warp's rays stay closer in position and direction.  TOP > 0:
// the top levels were staged in s_top by stage_top<TOP> (single-BVH sources
// only).  SPEC: speculative traversal
// (Aila and Laine 2009) — it changes the order in which a ray meets its
// nodes, so it is only for any-hit rays whose result is hit or miss alone
// (which triangle was found first is not reported by such sources).
// INLOOP: finish and refill inside the inner phase (above); leaf_batch: the
// parked leaves that end an INLOOP inner phase (1..32).  Neither changes a
// ray's order of nodes.
template <int ANY, bool MT, bool STATS, int STACK, int STRIDE, class Src, int CHUNK = int(kChunk), int TOP = 0,
          bool SPEC = false, bool INLOOP = false>
__device__ __forceinline__ void trace_persistent(const rq_bvh4_node* __restrict__ nodes,
                                                 const rq_triangle* __restrict__ tris, Src& src, uint32_t* ctr,
                                                 int32_t* stk, uint32_t* err, int stack_cap = STACK,
                                                 const float4* s_top = nullptr, int refill_min = 1,
                                                 int leaf_batch = 32) {
    static_assert(TOP == 0 || !IsMulti<Src>::value, "top-level staging needs one BVH per launch");
    static_assert(!SPEC || ANY == 1, "speculative traversal changes which hit an any-hit ray finds first");
    static_assert(!INLOOP || !HasRoundEnd<Src>::value, "in-loop refill reports rays outside the round hooks");
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    // warp-uniform chunk of ray ids
    uint32_t next = 0, end = 0;
    bool exhausted = false;
    // lane state
    bool active = false;
    uint32_t rid = 0;
    typename Src::Meta meta;
    Ray ray;
    SlabRay sr;
    WtRay w;
    float best = 0.0f;
    int sp = 0;            // entries in the shared-memory stack
    int32_t top = 0;       // the stack's top entry, kept in a register
    bool has_top = false;
    Hit h;
    h.hit = false;
    h.t = 0.0f;
    h.idx = kNoHit;
    h.u = h.v = 0.0f;
    h.boxes = h.tris = 0;

    int32_t leaf = kNoLeaf;  // the lane's parked leaf entry
    bool stalled = false;    // SPEC: a second leaf waits in `top`

    // hand the next ray ids to idle lanes once refill_min of them are idle
    // (called by all 32 lanes together)
    auto refill = [&]() {
        uint32_t idle = __ballot_sync(kFull, !active);
        const bool go = __popc(idle) >= refill_min || idle == kFull;
        while (go && idle && !exhausted) {
            if (next == end) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(ctr, uint32_t(CHUNK));
                base = __shfl_sync(kFull, base, 0);
                if (base >= src.total) {
                    exhausted = true;
                    break;
                }
                next = base;
                end = min(base + uint32_t(CHUNK), src.total);
            }
            const uint32_t take = min(uint32_t(__popc(idle)), end - next);
            const uint32_t rank = __popc(idle & lt_mask);
            const bool mine = ((idle >> lane) & 1u) && rank < take;
            if (mine) {
                rid = next + rank;
                if (src.make(rid, ray, meta)) {
                    active = true;
                    sr.ix = safe_inv(ray.d.x);
                    sr.iy = safe_inv(ray.d.y);
                    sr.iz = safe_inv(ray.d.z);
                    sr.ox = ray.o.x * sr.ix;
                    sr.oy = ray.o.y * sr.iy;
                    sr.oz = ray.o.z * sr.iz;
                    if (!MT) w = wt_setup(ray.d);
                    best = ray.tmax;
                    h.hit = false;
                    h.idx = kNoHit;
                    h.u = h.v = 0.0f;
                    h.boxes = h.tris = 0;
                    top = TOP > 0 ? kStaged : 0;  // the root (slot 0 when staged)
                    has_top = true;
                    sp = 0;
                    leaf = kNoLeaf;
                    stalled = false;
                }
            }
            next += take;
            // lanes whose id made no ray (a light behind the surface, an
            // empty pixel) take the next id at once
            idle = __ballot_sync(kFull, !active);
        }
    };

    for (;;) {
        // ---- refill idle lanes
        refill();
        if (!__any_sync(kFull, active)) {
            if (exhausted) break;
            continue;
        }

        // ---- inner phase (SPEC: lanes holding a leaf keep taking inner
        // nodes while other lanes still search; a second leaf stays on the
        // stack and stalls the lane until the leaf phase)
        leaf = kNoLeaf;
        stalled = false;
        for (;;) {
            if constexpr (INLOOP) {
                // a ray whose stack ran out with no leaf pending is done
                if (active && !(has_top || sp > 0) && leaf == kNoLeaf) {
                    h.t = best;
                    src.finish(rid, meta, ray, h);
                    active = false;
                }
                refill();
            }
            const bool left = has_top || sp > 0;
            const bool searching = active && left && leaf == kNoLeaf;
            if (!__any_sync(kFull, searching)) break;
            if constexpr (INLOOP) {
                if (__popc(__ballot_sync(kFull, active && leaf != kNoLeaf)) >= leaf_batch) break;
            }
            const bool want = SPEC ? (active && left && !stalled) : searching;
            if (!want) continue;
            int32_t e;
            if (has_top) {
                e = top;
                has_top = false;
            } else {
                e = stk[(--sp) * STRIDE];
            }
            if (e < 0) {
                if (!SPEC || leaf == kNoLeaf) {
                    leaf = e;
                } else {
                    top = e;
                    has_top = true;
                    stalled = true;
                }
                continue;
            }
            // box tests, each axis's near and far plane rows chosen by the
            // ray's signs
            float tk[4];
            uint32_t hitm;
            int4 cix, cnt;
            if (TOP > 0 && (e & kStaged)) {
                const float4* sp4 = s_top + (e & ~kStaged) * kTopStride;
                hitm = box4_nf<false>([&](int i) { return sp4[i]; }, sr, ray.tmin, best, tk);
                const float4 a = sp4[6], b = sp4[7];
                cix = make_int4(__float_as_int(a.x), __float_as_int(a.y), __float_as_int(a.z), __float_as_int(a.w));
                cnt = make_int4(__float_as_int(b.x), __float_as_int(b.y), __float_as_int(b.z), __float_as_int(b.w));
            } else {
                const rq_bvh4_node* nb = IsMulti<Src>::value ? ray.nodes : nodes;
                const float4* np = reinterpret_cast<const float4*>(nb + e);
                hitm = box4_nf<false>([&](int i) { return ldg4(np + i); }, sr, ray.tmin, best, tk);
                cix = ldg4i(reinterpret_cast<const int4*>(np + 6));
                cnt = ldg4i(reinterpret_cast<const int4*>(np + 7));
            }
            if (STATS) h.boxes += 4;
            const int32_t aci[4] = {cix.x, cix.y, cix.z, cix.w}, acc[4] = {cnt.x, cnt.y, cnt.z, cnt.w};
            // closest hit: near to far; any hit: slot order.  The first child
            // to visit stays in the register.
            if (ANY == 1 || (ANY == kAnyPerRay && ray.any))
                push_children_any<STRIDE>(hitm, aci, acc, stk, sp, stack_cap, top, has_top, err, RQ_DERR_STACK);
            else
                push_children<STRIDE>(hitm, aci, acc, tk, true, stk, sp, stack_cap, top, has_top, err, RQ_DERR_STACK);
        }

        // ---- leaf phase
        bool done = false;
        if (active && leaf != kNoLeaf) {
            const uint32_t first = uint32_t(leaf) & 0x07ffffffu;
            const uint32_t cntl = ((uint32_t(leaf) >> 27) & 15u) + 1u;
            for (uint32_t p = first; p < first + cntl; ++p) {
                const float4* tp = reinterpret_cast<const float4*>((IsMulti<Src>::value ? ray.tris : tris) + p);
                const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
                const F3 v0{a.x, a.y, a.z}, v1{b.x, b.y, b.z}, v2{c.x, c.y, c.z};
                if (STATS) ++h.tris;
                float t, u, v;
                const bool ok = MT ? mt_test(ray.o, ray.d, v0, v1, v2, 1e-7f, t, u, v)
                                   : wt_test(w, ray.o, v0, v1, v2, t, u, v);
                if (ok && t >= ray.tmin && t < best) {
                    best = t;
                    h.hit = true;
                    h.idx = p;
                    h.u = u;
                    h.v = v;
                    if (ANY == 1 || (ANY == kAnyPerRay && ray.any)) {
                        done = true;
                        break;
                    }
                }
            }
        }

        // ---- report finished rays
        bool fin = false;
        if (active && (done || (sp == 0 && !has_top))) {
            h.t = best;
            src.finish(rid, meta, ray, h);
            active = false;
            fin = true;
        }
        if constexpr (HasRoundEnd<Src>::value) {
            __syncwarp();
            src.round_end(fin, meta);
        }
    }
}

}  // namespace rq
