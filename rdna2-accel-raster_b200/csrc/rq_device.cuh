// rq_device.cuh — device helpers shared by the kernels: memory-ordering
// primitives, ordered-float encoding, the slab test, the two ray-triangle
// tests and the hash/trigonometry used by the ray generators.
//
// All float arithmetic follows IEEE single precision with one rounding per
// operation: the library is compiled with -fmad=false and fused operations
// are written explicitly (__fmaf_rn), so results are reproducible bit for bit
// by a CPU implementation of the same formulas.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/rq_layouts.h"

namespace rq {

// Primitive index of "no hit".
constexpr uint32_t kNoHit = 0xffffffffu;

// ------------------------------------------------------------ memory order
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Fetch-and-add with acquire-release semantics: releases this thread's
// earlier stores and acquires those released by earlier adds on the same
// word (the hand-off of a bottom-up refit, without separate fences).
template <bool CTA = false>
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    if (CTA)
        asm volatile("atom.acq_rel.cta.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    else
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
// L2-coherent 16-B load (bypasses L1), for data written by other blocks in
// the same launch.
__device__ __forceinline__ float4 ld_cg4(const float4* p) { return __ldcg(p); }

// Non-coherent read-only 16-B load through the texture path.
__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ int4 ldg4i(const int4* p) { return __ldg(p); }

// ---------------------------------------------------------- ordered floats
// Monotone map float -> uint32 (-inf < ... < -0 < +0 < ... < +inf).
__device__ __forceinline__ uint32_t f2o(float f) {
    uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// ------------------------------------------------------------------ Morton
__device__ __forceinline__ uint32_t expand10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
__device__ __forceinline__ uint32_t quantize10(float c, float lo, float scale) {
    float t = (c - lo) * scale;
    if (t >= 1023.0f) return 1023u;
    if (t > 0.0f) return (uint32_t)t;
    return 0u;
}

// --------------------------------------------------------------- slab test
#define RQ_TWO_POW_100 1.2676506002282294e30f
#define RQ_TWO_POW_M100 7.888609052210118e-31f
#define RQ_FAR_SCALE 1.00000095367431640625f

// 1/d, with |d| < 2^-100 replaced by a signed 2^100 so o*inv stays exact.
__device__ __forceinline__ float safe_inv(float d) {
    return fabsf(d) < RQ_TWO_POW_M100 ? copysignf(RQ_TWO_POW_100, d) : 1.0f / d;
}

struct SlabRay {
    float ix, iy, iz;  // inverse direction
    float ox, oy, oz;  // origin * inverse direction
};

__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Entry distance and hit flag of one box: fused (b*inv - o*inv) plane
// distances, entry clamped below by tmin, exit above by best, exit widened
// by 2^-20 relative.
__device__ __forceinline__ bool slab(const SlabRay& r, float tmin, float best, float mnx, float mxx, float mny,
                                     float mxy, float mnz, float mxz, float& tn) {
    float tx0 = __fmaf_rn(mnx, r.ix, -r.ox), tx1 = __fmaf_rn(mxx, r.ix, -r.ox);
    float ty0 = __fmaf_rn(mny, r.iy, -r.oy), ty1 = __fmaf_rn(mxy, r.iy, -r.oy);
    float tz0 = __fmaf_rn(mnz, r.iz, -r.oz), tz1 = __fmaf_rn(mxz, r.iz, -r.oz);
    float a = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    float b = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), best));
    tn = a;
    return a <= b * RQ_FAR_SCALE;
}

// Two IEEE single-precision operations per instruction (the packed f32x2
// forms of sm_100); each lane is one rounding, as the scalar form.
__device__ __forceinline__ unsigned long long pack2(float a, float b) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 unpack2(unsigned long long r) {
    float2 v;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(v.x), "=f"(v.y) : "l"(r));
    return v;
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b,
                                                    unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned long long fmul2(unsigned long long a, unsigned long long b) {
    unsigned long long d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// Plane distances b*inv - o*inv of the 4 children on one axis, two children
// per packed fused multiply-add.
__device__ __forceinline__ void planes4(float4 b, float inv, float oinv, float (&t)[4]) {
    const unsigned long long i2 = pack2(inv, inv), o2 = pack2(-oinv, -oinv);
    const float2 lo = unpack2(ffma2(pack2(b.x, b.y), i2, o2)), hi = unpack2(ffma2(pack2(b.z, b.w), i2, o2));
    t[0] = lo.x;
    t[1] = lo.y;
    t[2] = hi.x;
    t[3] = hi.y;
}

// Rows of a node in global memory, for box4_nf.
struct GlobalRows {
    const float4* np;
    __device__ __forceinline__ float4 operator()(int i) const { return __ldg(np + i); }
};

// The slab test of the 4 children of one 4-wide node, one axis at a time, so
// that only one axis's two plane rows are held at once.  `row(i)` returns row
// i of the node (16 B: min_x, max_x, min_y, max_y, min_z, max_z, child_index,
// child_count).  Each axis's near plane is picked by the sign of the inverse
// direction (the max row when it is negative): b*inv - o*inv, one rounding, is
// monotonic in b, so for every box with min <= max the near plane's distance
// is the smaller of the pair, and entry and exit equal slab()'s (up to the
// sign of a zero entry, which no comparison sees); boxes with min > max on an
// axis are empty here.  Entry max(near_x, near_y, near_z, tmin), exit
// min(far_x, far_y, far_z, best) widened by 2^-20 relative, with sm_100's
// three-input min/max.  Returns the hit mask (bit k: slot k non-empty and
// hit) and the entry distances in tk.  PACKED: plane distances two per packed
// instruction (measured faster for the one-ray-per-thread camera traversal,
// slower in the persistent engine).
template <bool PACKED, class Row>
__device__ __forceinline__ uint32_t box4_nf(Row row, const SlabRay& r, float tmin, float best, float (&tk)[4]) {
    auto planes = [](float4 b, float inv, float oinv, float (&t)[4]) {
        if (PACKED) {
            planes4(b, inv, oinv, t);
        } else {
            t[0] = __fmaf_rn(b.x, inv, -oinv);
            t[1] = __fmaf_rn(b.y, inv, -oinv);
            t[2] = __fmaf_rn(b.z, inv, -oinv);
            t[3] = __fmaf_rn(b.w, inv, -oinv);
        }
    };
    // near-plane rows from the signs (recomputed per node: fewer live registers)
    const int nx = int(__float_as_uint(r.ix) >> 31), ny = 2 + int(__float_as_uint(r.iy) >> 31),
              nz = 4 + int(__float_as_uint(r.iz) >> 31);
    float tf[4];
    planes(row(nx), r.ix, r.ox, tk);
    planes(row(nx ^ 1), r.ix, r.ox, tf);
    {
        float an[4], af[4];
        planes(row(ny), r.iy, r.oy, an);
        planes(row(ny ^ 1), r.iy, r.oy, af);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            tk[k] = fmaxf(tk[k], an[k]);
            tf[k] = fminf(tf[k], af[k]);
        }
    }
    {
        float an[4], af[4];
        planes(row(nz), r.iz, r.oz, an);
        planes(row(nz ^ 1), r.iz, r.oz, af);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            tk[k] = fmax3(tk[k], an[k], tmin);
            tf[k] = fmin3(tf[k], af[k], best);
        }
    }
    const float4 c = row(7);
    const int32_t cc[4] = {__float_as_int(c.x), __float_as_int(c.y), __float_as_int(c.z), __float_as_int(c.w)};
    uint32_t hitm = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (cc[k] != 0 && tk[k] <= tf[k] * RQ_FAR_SCALE) hitm |= 1u << k;
    return hitm;
}

// ------------------------------------------------------- triangle tests
struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float f3dot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ F3 f3cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ F3 f3norm(F3 v) {
    float len = sqrtf(f3dot(v, v));
    return {v.x / len, v.y / len, v.z / len};
}
__device__ __forceinline__ float f3c(F3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Moller-Trumbore in the arithmetic of software_bvh_bvh4.comp:166-178.
__device__ __forceinline__ bool mt_test(F3 o, F3 d, F3 v0, F3 v1, F3 v2, float eps, float& t, float& u,
                                        float& v) {
    F3 e1 = f3sub(v1, v0);
    F3 e2 = f3sub(v2, v0);
    F3 h = f3cross(d, e2);
    float a = f3dot(e1, h);
    if (fabsf(a) < eps) return false;
    float f = 1.0f / a;
    F3 s = f3sub(o, v0);
    u = f * f3dot(s, h);
    if (u < 0.0f || u > 1.0f) return false;
    F3 q = f3cross(s, e1);
    v = f * f3dot(d, q);
    if (v < 0.0f || u + v > 1.0f) return false;
    t = f * f3dot(e2, q);
    return true;
}

// Watertight test (Woop, Benthin, Wald 2013) with per-ray shear constants.
struct WtRay {
    int kx, ky, kz;
    float sx, sy, sz;
};

__device__ __forceinline__ WtRay wt_setup(F3 d) {
    WtRay w;
    float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int kz = 0;
    float m = ax;
    if (ay > m) {
        kz = 1;
        m = ay;
    }
    if (az > m) kz = 2;
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    float dz = f3c(d, kz);
    if (dz < 0.0f) {
        int t = kx;
        kx = ky;
        ky = t;
    }
    w.kx = kx;
    w.ky = ky;
    w.kz = kz;
    w.sx = f3c(d, kx) / dz;
    w.sy = f3c(d, ky) / dz;
    w.sz = 1.0f / dz;
    return w;
}

// Shared-edge edge functions are exact negations of each other (plain float
// products), exact zeros are re-evaluated in double, t = T / det rounded once.
// KX, KY, KZ: the ray's permuted axes fixed at compile time (no per-vertex
// component selection); -1: taken from w at run time.
template <int KX, int KY, int KZ>
__device__ __forceinline__ bool wt_test_k(const WtRay& w, F3 o, F3 v0, F3 v1, F3 v2, float& t, float& u, float& v) {
    const int kx = KX < 0 ? w.kx : KX, ky = KY < 0 ? w.ky : KY, kz = KZ < 0 ? w.kz : KZ;
    F3 A = f3sub(v0, o), B = f3sub(v1, o), C = f3sub(v2, o);
    float Az0 = f3c(A, kz), Bz0 = f3c(B, kz), Cz0 = f3c(C, kz);
    float Ax = __fmaf_rn(-w.sx, Az0, f3c(A, kx));
    float Ay = __fmaf_rn(-w.sy, Az0, f3c(A, ky));
    float Bx = __fmaf_rn(-w.sx, Bz0, f3c(B, kx));
    float By = __fmaf_rn(-w.sy, Bz0, f3c(B, ky));
    float Cx = __fmaf_rn(-w.sx, Cz0, f3c(C, kx));
    float Cy = __fmaf_rn(-w.sy, Cz0, f3c(C, ky));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
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

__device__ __forceinline__ bool wt_test(const WtRay& w, F3 o, F3 v0, F3 v1, F3 v2, float& t, float& u, float& v) {
    return wt_test_k<-1, -1, -1>(w, o, v0, v1, v2, t, u, v);
}

// The same test through one of the six fixed-axis forms, chosen per ray (the
// rays of a warp mostly share one): fewer instructions per triangle, more
// code.  Faster for the one-ray-per-thread camera traversal, not in the
// persistent engine.
__device__ __forceinline__ bool wt_test_fixed(const WtRay& w, F3 o, F3 v0, F3 v1, F3 v2, float& t, float& u,
                                              float& v) {
    if (w.kz == 2)
        return w.kx == 0 ? wt_test_k<0, 1, 2>(w, o, v0, v1, v2, t, u, v)
                         : wt_test_k<1, 0, 2>(w, o, v0, v1, v2, t, u, v);
    if (w.kz == 1)
        return w.kx == 2 ? wt_test_k<2, 0, 1>(w, o, v0, v1, v2, t, u, v)
                         : wt_test_k<0, 2, 1>(w, o, v0, v1, v2, t, u, v);
    return w.kx == 1 ? wt_test_k<1, 2, 0>(w, o, v0, v1, v2, t, u, v) : wt_test_k<2, 1, 0>(w, o, v0, v1, v2, t, u, v);
}

// ------------------------------------------------------------------ hashes
__host__ __device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
#define RQ_INV_2POW32 2.3283064365386963e-10f
__device__ __forceinline__ float hash_float(uint32_t seed) { return __uint2float_rn(pcg_hash(seed)) * RQ_INV_2POW32; }

// One-at-a-time style hash of shaders/rq_ao.comp:18-25.
__device__ __forceinline__ uint32_t ao_hash(uint32_t x) {
    x += (x << 10u);
    x ^= (x >> 6u);
    x += (x << 3u);
    x ^= (x >> 11u);
    x += (x << 15u);
    return x;
}

// sin and cos from a Cody-Waite reduction by pi/2 (three-part constant) and
// Taylor polynomials with coefficients 1/n! on [-pi/4, pi/4], evaluated with
// explicit fused multiply-adds.  Used where the generated rays must be
// reproducible bit for bit on the CPU.
__device__ __forceinline__ void sincos_taylor(float x, float* s, float* c) {
    float n = floorf(__fmaf_rn(x, 0x1.45f306p-1f, 0.5f));
    float r = __fmaf_rn(-n, 0x1.921fb6p+0f, x);
    r = __fmaf_rn(-n, -0x1.777a5cp-25f, r);
    r = __fmaf_rn(-n, -0x1.ee59dap-50f, r);
    float r2 = r * r;
    float ps = __fmaf_rn(r2, 0x1.71de3ap-19f, -0x1.a01a02p-13f);
    ps = __fmaf_rn(r2, ps, 0x1.111112p-7f);
    ps = __fmaf_rn(r2, ps, -0x1.555556p-3f);
    ps = __fmaf_rn(r2 * r, ps, r);
    float pc = __fmaf_rn(r2, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = __fmaf_rn(r2, pc, -0x1.6c16c2p-10f);
    pc = __fmaf_rn(r2, pc, 0x1.555556p-5f);
    pc = __fmaf_rn(r2, pc, -0.5f);
    pc = __fmaf_rn(r2, pc, 1.0f);
    int q = (int)((long long)n & 3);
    *s = q == 0 ? ps : (q == 1 ? pc : (q == 2 ? -ps : -pc));
    *c = q == 0 ? pc : (q == 1 ? -ps : (q == 2 ? -pc : ps));
}

// Cosine-weighted direction about the unit normal N from two draws in [0,1]
// (the hemisphere sample of shaders/rq_ao.comp:32-45: r = sqrt(u1),
// theta = 2 pi u2, tangent frame from the cross product with z or x).
__device__ __forceinline__ F3 cosine_hemisphere(F3 N, float u1, float u2) {
    const float r = sqrtf(u1);
    const float theta = 6.2831853f * u2;
    float sn, cs;
    sincos_taylor(theta, &sn, &cs);
    const float x = r * cs, y = r * sn, z = sqrtf(fmaxf(0.0f, 1.0f - u1));
    const F3 up = fabsf(N.z) < 0.999f ? F3{0.0f, 0.0f, 1.0f} : F3{1.0f, 0.0f, 0.0f};
    const F3 tg = f3norm(f3cross(up, N));
    const F3 bt = f3cross(N, tg);
    return f3norm(F3{(tg.x * x + bt.x * y) + N.x * z, (tg.y * x + bt.y * y) + N.y * z,
                     (tg.z * x + bt.z * y) + N.z * z});
}

// ------------------------------------------------------------ bounded wait
// Iteration cap for spin-waits on flags written by other blocks of the same
// launch: with __nanosleep(64) it is several seconds, far beyond any
// legitimate wait, after which the waiter records an error and moves on.
#define RQ_SPIN_LIMIT (1u << 26)

__device__ __forceinline__ void set_err(uint32_t* err, uint32_t bit) { atomicOr(err, bit); }

// Wait until *p (read with acquire) differs from v: at most `limit` polls,
// 64 ns apart.  On giving up, sets `bit` in the error word and returns false.
__device__ __forceinline__ bool wait_change(const uint32_t* p, uint32_t v, uint32_t limit, uint32_t* err,
                                            uint32_t bit) {
    for (uint32_t spins = 0; ld_acquire(p) == v;) {
        if (++spins > limit) {
            set_err(err, bit);
            return false;
        }
        __nanosleep(64);
    }
    return true;
}

// ------------------------------------------------------ 4-wide child push
// Push the hit children of one 4-wide node (bit k of `hitm`: slot k hit, with
// entry distance tk[k]; child_index ci[k] and child_count cc[k] as stored in
// the node give its stack entry: the node index for an inner child, else
// bit31 | (count-1) << 27 | first primitive) so that they pop in visit
// order: ascending (tk, slot) when `sorted` (closest hit), ascending slot
// otherwise.  The first child to visit goes to the register `top`, the rest
// onto the shared-memory column `stk` (STRIDE words apart).  Each child's
// place is its rank among the hits, so nothing is indexed by a run-time
// value in registers.  With more hits than room (sp + hits > cap),
// `overflow_bit` is set in the error word and only the first cap - sp
// children in visit order are kept.
template <int STRIDE>
__device__ __forceinline__ void push_children(uint32_t hitm, const int32_t (&ci)[4], const int32_t (&cc)[4],
                                              const float (&tk)[4],
                                              bool sorted, int32_t* stk, int& sp, int cap, int32_t& top,
                                              bool& has_top, uint32_t* err, uint32_t overflow_bit) {
    int nh = __popc(hitm);
    if (sp + nh > cap) {
        set_err(err, overflow_bit);
        nh = max(cap - sp, 0);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!((hitm >> k) & 1u)) continue;
        int rank;
        if (sorted) {
            rank = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (j == k) continue;
                const bool before = j < k ? tk[j] <= tk[k] : tk[j] < tk[k];
                rank += int(((hitm >> j) & 1u) && before);
            }
        } else {
            rank = __popc(hitm & ((1u << k) - 1u));
        }
        const int32_t ent = cc[k] < 0 ? ci[k] : int32_t(0x80000000u | (uint32_t(cc[k] - 1) << 27) | uint32_t(~ci[k]));
        if (rank == 0) {
            if (nh > 0) {
                top = ent;
                has_top = true;
            }
        } else if (rank < nh) {
            stk[(sp + nh - 1 - rank) * STRIDE] = ent;
        }
    }
    if (nh > 0) sp += nh - 1;
}

// Any-hit form of push_children (slot order, no distances): the hit slots
// are walked from slot 3 down, each pushed when a lower hit slot follows, so
// the lowest hit slot ends in `top`.
template <int STRIDE>
__device__ __forceinline__ void push_children_any(uint32_t hitm, const int32_t (&ci)[4], const int32_t (&cc)[4],
                                                  int32_t* stk, int& sp, int cap, int32_t& top, bool& has_top,
                                                  uint32_t* err, uint32_t overflow_bit) {
    const int nh = __popc(hitm);
    if (sp + nh > cap) {
        set_err(err, overflow_bit);
        const int keep = max(cap - sp, 0);
        while (__popc(hitm) > keep) hitm &= ~(0x80000000u >> __clz(hitm));  // drop the highest slot
    }
    bool pending = false;
    int32_t pend = 0;
#pragma unroll
    for (int k = 3; k >= 0; --k) {
        if (!((hitm >> k) & 1u)) continue;
        if (pending) stk[(sp++) * STRIDE] = pend;
        pend = cc[k] < 0 ? ci[k] : int32_t(0x80000000u | (uint32_t(cc[k] - 1) << 27) | uint32_t(~ci[k]));
        pending = true;
    }
    if (pending) {
        top = pend;
        has_top = true;
    }
}

}  // namespace rq
