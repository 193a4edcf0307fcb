// k_tlas.cu — two-level scenes: instances of BLAS handles, each with an
// object-to-world transform and an instance id, under a top-level BVH (the
// instance acceleration structures the reference builds through the driver,
// common/vk_bvh.cpp:237-336, with the VkAccelerationStructureInstanceKHR
// records of benchmarks/exp1_visbuf/visbuf_main.cpp:762-771).
//
//  k_instance_boxes  world box of each instance: the BLAS root node's slot
//                    boxes united, its 8 corners transformed, widened by
//                    2^-20 of the coordinate magnitudes (rounding of the
//                    transform must not shrink it); written as the
//                    degenerate triangle (min, max, min), whose bounds are
//                    exactly the box, so the LBVH build of rq_build makes
//                    the top-level tree (one instance per leaf).
//  k_trace_tlas      one ray per thread.  The stack holds top-level entries;
//                    at an instance leaf the ray is moved into object space
//                    (origin and direction by the inverse transform, the
//                    direction not renormalised, so t is the same in both
//                    spaces and one best-t serves all instances), a marker
//                    entry is pushed and then the BLAS root; popping the
//                    marker returns to world space.  Closest hit sorts
//                    children near-to-far at both levels.
#include "rq_device.cuh"
#include "rq_internal.h"
#include "rq_tlas.h"

namespace {

using namespace rq;

constexpr int kTT = 128;
constexpr int32_t kMarker = 0x40000000;  // "leave the instance" (inner entries are < 2^27)

__global__ void __launch_bounds__(128) k_instance_boxes(const TlasInst* __restrict__ inst,
                                                        const float* __restrict__ fwd, uint32_t n,
                                                        float* __restrict__ tri9) {
    const uint32_t i = blockIdx.x * 128u + threadIdx.x;
    if (i >= n) return;
    const float4* np = reinterpret_cast<const float4*>(inst[i].nodes);
    const float4 mnx = np[0], mxx = np[1], mny = np[2], mxy = np[3], mnz = np[4], mxz = np[5];
    const int4 cnt = reinterpret_cast<const int4*>(np)[7];
    const float amnx[4] = {mnx.x, mnx.y, mnx.z, mnx.w}, amxx[4] = {mxx.x, mxx.y, mxx.z, mxx.w};
    const float amny[4] = {mny.x, mny.y, mny.z, mny.w}, amxy[4] = {mxy.x, mxy.y, mxy.z, mxy.w};
    const float amnz[4] = {mnz.x, mnz.y, mnz.z, mnz.w}, amxz[4] = {mxz.x, mxz.y, mxz.z, mxz.w};
    const int32_t acc[4] = {cnt.x, cnt.y, cnt.z, cnt.w};
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 4; ++k) {
        if (acc[k] == 0) continue;
        lo[0] = fminf(lo[0], amnx[k]);
        lo[1] = fminf(lo[1], amny[k]);
        lo[2] = fminf(lo[2], amnz[k]);
        hi[0] = fmaxf(hi[0], amxx[k]);
        hi[1] = fmaxf(hi[1], amxy[k]);
        hi[2] = fmaxf(hi[2], amxz[k]);
    }
    const float* f = fwd + 12ull * i;
    float wlo[3] = {INFINITY, INFINITY, INFINITY}, whi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 8; ++c) {
        const float x = (c & 1) ? hi[0] : lo[0], y = (c & 2) ? hi[1] : lo[1], z = (c & 4) ? hi[2] : lo[2];
        for (int r = 0; r < 3; ++r) {
            const float w = ((f[4 * r] * x + f[4 * r + 1] * y) + f[4 * r + 2] * z) + f[4 * r + 3];
            wlo[r] = fminf(wlo[r], w);
            whi[r] = fmaxf(whi[r], w);
        }
    }
    float* t = tri9 + 9ull * i;
    for (int r = 0; r < 3; ++r) {
        const float pad = (fabsf(wlo[r]) + fabsf(whi[r])) * 0x1p-20f;
        const float a = wlo[r] - pad, b = whi[r] + pad;
        t[r] = a;
        t[3 + r] = b;
        t[6 + r] = a;
    }
}

__device__ __forceinline__ SlabRay slab_setup(F3 o, F3 d) {
    SlabRay sr;
    sr.ix = safe_inv(d.x);
    sr.iy = safe_inv(d.y);
    sr.iz = safe_inv(d.z);
    sr.ox = o.x * sr.ix;
    sr.oy = o.y * sr.iy;
    sr.oz = o.z * sr.iz;
    return sr;
}

template <bool ANY, bool MT>
__global__ void __launch_bounds__(kTT) k_trace_tlas(const rq_bvh4_node* __restrict__ top,
                                                    const uint32_t* __restrict__ top_perm,
                                                    const TlasInst* __restrict__ inst, const rq_ray* __restrict__ rays,
                                                    uint32_t n, uint32_t cull, rq_hit* __restrict__ hits, int stack_cap,
                                                    uint32_t* err) {
    extern __shared__ int32_t s_stack[];
    const uint32_t id = blockIdx.x * kTT + threadIdx.x;
    if (id >= n) return;
    int32_t* stk = s_stack + threadIdx.x;
    const float4* rp = reinterpret_cast<const float4*>(rays + id);
    const float4 r0 = __ldg(rp), r1 = __ldg(rp + 1);
    const F3 o{r0.x, r0.y, r0.z}, d{r1.x, r1.y, r1.z};
    const float tmin = r0.w;
    float best = r1.w;
    const SlabRay world = slab_setup(o, d);
    SlabRay sr = world;
    F3 oo = o, od = d;  // the ray in the current instance's space
    WtRay w = wt_setup(d);
    bool inside = false;
    const rq_bvh4_node* nodes = top;
    const rq_triangle* tris = nullptr;
    const uint32_t* perm = nullptr;
    uint32_t cur_id = 0;
    uint32_t hit_inst = 0xffffffffu, hit_prim = 0xffffffffu;
    bool hit = false;
    stk[0] = 0;
    int sp = 1;
    bool done = false;
    while (sp > 0 && !done) {
        const int32_t e = stk[(--sp) * kTT];
        if (e == kMarker) {  // back to the top level
            inside = false;
            nodes = top;
            sr = world;
            continue;
        }
        if (e >= 0) {
            const float4* np = reinterpret_cast<const float4*>(nodes + e);
            float tk[4];
            const uint32_t hitm = box4_nf<false>(GlobalRows{np}, sr, tmin, best, tk);
            const int4 cix = ldg4i(reinterpret_cast<const int4*>(np + 6));
            const int4 cnt = ldg4i(reinterpret_cast<const int4*>(np + 7));
            const int32_t aci[4] = {cix.x, cix.y, cix.z, cix.w}, acc[4] = {cnt.x, cnt.y, cnt.z, cnt.w};
            // the first child to visit comes back as `first`; here it goes on
            // top of the shared-memory stack with the others
            int32_t first = 0;
            bool has_first = false;
            if (ANY)
                push_children_any<kTT>(hitm, aci, acc, stk, sp, stack_cap, first, has_first, err, RQ_DERR_STACK);
            else
                push_children<kTT>(hitm, aci, acc, tk, true, stk, sp, stack_cap, first, has_first, err,
                                   RQ_DERR_STACK);
            if (has_first) stk[(sp++) * kTT] = first;
            continue;
        }
        const uint32_t first = uint32_t(e) & 0x07ffffffu;
        const uint32_t cntl = ((uint32_t(e) >> 27) & 15u) + 1u;
        if (!inside) {  // an instance (one per top-level leaf)
            const TlasInst* in = inst + __ldg(top_perm + first);
            if ((__ldg(&in->mask) & cull) == 0u) continue;
            float m[12];
#pragma unroll
            for (int k = 0; k < 12; ++k) m[k] = __ldg(&in->inv[k]);
            oo = F3{((m[0] * o.x + m[1] * o.y) + m[2] * o.z) + m[3], ((m[4] * o.x + m[5] * o.y) + m[6] * o.z) + m[7],
                    ((m[8] * o.x + m[9] * o.y) + m[10] * o.z) + m[11]};
            od = F3{(m[0] * d.x + m[1] * d.y) + m[2] * d.z, (m[4] * d.x + m[5] * d.y) + m[6] * d.z,
                    (m[8] * d.x + m[9] * d.y) + m[10] * d.z};
            sr = slab_setup(oo, od);
            if (!MT) w = wt_setup(od);
            nodes = in->nodes;
            tris = in->tris;
            perm = in->perm;
            cur_id = __ldg(&in->instance_id);
            inside = true;
            if (sp + 2 > stack_cap) {
                set_err(err, RQ_DERR_STACK);
                break;
            }
            stk[(sp++) * kTT] = kMarker;
            stk[(sp++) * kTT] = 0;
            continue;
        }
        for (uint32_t p = first; p < first + cntl; ++p) {
            const float4* tp = reinterpret_cast<const float4*>(tris + p);
            const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
            const F3 v0{a.x, a.y, a.z}, v1{b.x, b.y, b.z}, v2{c.x, c.y, c.z};
            float t, u, v;
            const bool ok = MT ? mt_test(oo, od, v0, v1, v2, 1e-7f, t, u, v) : wt_test(w, oo, v0, v1, v2, t, u, v);
            if (ok && t >= tmin && t < best) {
                best = t;
                hit = true;
                hit_inst = cur_id;
                hit_prim = __ldg(perm + p);
                if (ANY) {
                    done = true;
                    break;
                }
            }
        }
    }
    uint4 out = make_uint4(0u, __float_as_uint(-1.0f), 0xffffffffu, 0xffffffffu);
    if (hit) out = make_uint4(1u, __float_as_uint(best), hit_inst, hit_prim);
    reinterpret_cast<uint4*>(hits)[id] = out;
}

}  // namespace

int rq_launch_instance_boxes(rq_ctx* ctx, const TlasInst* inst, const float* fwd, uint32_t n, float* tri9,
                             cudaStream_t st) {
    k_instance_boxes<<<(n + 127) / 128, 128, 0, st>>>(inst, fwd, n, tri9);
    return rq_cuda_status(ctx, cudaGetLastError(), "instance boxes launch");
}

int rq_launch_trace_tlas(rq_ctx* ctx, const rq_tlas* t, const rq_ray* rays, uint32_t n, uint32_t flags,
                         uint32_t cull_mask, rq_hit* hits, cudaStream_t st) {
    if (n == 0) return RQ_OK;
    const bool any = flags & RQ_TRACE_ANY, mt = flags & RQ_TRI_MT;
    const int stack = int((t->stack_bound + 3u) & ~3u);
    const size_t smem = size_t(stack) * kTT * sizeof(int32_t);
    auto k = any ? (mt ? k_trace_tlas<true, true> : k_trace_tlas<true, false>)
                 : (mt ? k_trace_tlas<false, true> : k_trace_tlas<false, false>);
    cudaError_t e = cudaSuccess;
    if (smem > 48 * 1024) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e == cudaSuccess) {
        k<<<(n + kTT - 1) / kTT, kTT, smem, st>>>(t->top->nodes4, t->top->perm, t->d_inst, rays, n, cull_mask, hits,
                                                   stack, ctx->d_err);
        e = cudaGetLastError();
    }
    return rq_cuda_status(ctx, e, "tlas trace launch");
}
