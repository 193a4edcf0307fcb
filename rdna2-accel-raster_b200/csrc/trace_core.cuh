// trace_core.cuh — the engine's 4-wide traversal of one ray by one thread
// from start to end (the schedule for one coherent ray per thread, such as
// camera rays; trace_engine.cuh is the schedule that refills lanes).
//
// Stack entries are int32: >= 0 an inner node index; bit 31 set a leaf
// (bits 27..30 = count-1, bits 0..26 = first primitive).  Each thread's
// stack lives in shared memory with a stride of the block size, so the
// entries of one warp fall in distinct banks.  3*depth+1 entries suffice.
// The visit order is the one of trace_engine.cuh: results are identical.
#pragma once

#include "rq_device.cuh"
#include "rq_internal.h"

namespace rq {

constexpr uint32_t kLeafBit = 0x80000000u;

struct TraceResult {
    float t;        // nearest accepted distance (tmax when nothing was hit)
    uint32_t idx;   // leaf-order primitive index, kNoHit for a miss
    float u, v;     // barycentrics of v1 and v2
    uint32_t boxes; // 4 per inner node visited
    uint32_t tris;  // triangles tested
};

// stack_cap: rows of the stack column actually allocated (at most STACK).
template <bool ANY, bool MT, bool STATS, int STACK, int STRIDE>
__device__ __forceinline__ void trace_ray(const rq_bvh4_node* __restrict__ nodes,
                                          const rq_triangle* __restrict__ tris, int32_t* stk, F3 o, F3 d,
                                          float tmin, float tmax, TraceResult& res, uint32_t* err,
                                          int stack_cap = STACK) {
    SlabRay sr;
    sr.ix = safe_inv(d.x);
    sr.iy = safe_inv(d.y);
    sr.iz = safe_inv(d.z);
    sr.ox = o.x * sr.ix;
    sr.oy = o.y * sr.iy;
    sr.oz = o.z * sr.iz;
    WtRay w;
    if (!MT) w = wt_setup(d);
    float best = tmax;
    res.idx = kNoHit;
    res.u = res.v = 0.0f;
    res.boxes = res.tris = 0;
    // the stack's top entry lives in a register: the nearest child of a node
    // is visited next without a round trip through shared memory
    int32_t top = 0;
    bool has_top = true;
    int sp = 0;
    while (has_top || sp > 0) {
        int32_t e;
        if (has_top) {
            e = top;
            has_top = false;
        } else {
            e = stk[(--sp) * STRIDE];
        }
        if (e >= 0) {
            const float4* np = reinterpret_cast<const float4*>(nodes + e);
            // box tests, each axis's near and far plane rows chosen by the
            // ray's signs
            float tk[4];
            const uint32_t hitm = box4_nf<true>([&](int i) { return ldg4(np + i); }, sr, tmin, best, tk);
            const int4 cix = ldg4i(reinterpret_cast<const int4*>(np + 6));
            const int4 cnt = ldg4i(reinterpret_cast<const int4*>(np + 7));
            if (STATS) res.boxes += 4;
            const int32_t aci[4] = {cix.x, cix.y, cix.z, cix.w}, acc[4] = {cnt.x, cnt.y, cnt.z, cnt.w};
            if (ANY)
                push_children_any<STRIDE>(hitm, aci, acc, stk, sp, stack_cap, top, has_top, err, RQ_DERR_STACK);
            else
                push_children<STRIDE>(hitm, aci, acc, tk, true, stk, sp, stack_cap, top, has_top, err, RQ_DERR_STACK);
        } else {
            const uint32_t first = uint32_t(e) & 0x07ffffffu;
            const uint32_t cntl = ((uint32_t(e) >> 27) & 15u) + 1u;
            bool done = false;
            for (uint32_t p = first; p < first + cntl; ++p) {
                const float4* tp = reinterpret_cast<const float4*>(tris + p);
                const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
                const F3 v0{a.x, a.y, a.z}, v1{b.x, b.y, b.z}, v2{c.x, c.y, c.z};
                if (STATS) ++res.tris;
                float t, u, v;
                const bool ok = MT ? mt_test(o, d, v0, v1, v2, 1e-7f, t, u, v) : wt_test_fixed(w, o, v0, v1, v2, t, u, v);
                if (ok && t >= tmin && t < best) {
                    best = t;
                    res.idx = p;
                    res.u = u;
                    res.v = v;
                    if (ANY) {
                        done = true;
                        break;
                    }
                }
            }
            if (ANY && done) break;
        }
    }
    res.t = best;
}

}  // namespace rq
