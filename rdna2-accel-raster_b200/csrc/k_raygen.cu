// k_raygen.cu — ray generators and the per-frame vertex deformation.
//
//  k_gen_procedural  software_bvh_bvh4.comp:60-94: coherent camera grid
//                    (1024 wide, x0.55 field) or PCG-hashed incoherent rays,
//                    tmin 0.01 and tmax 1000 (the shader's rayTMin / hitT).
//  k_deform_wave     z = base.z + amp*sin(t + freq*x) per vertex (the role of
//                    benchmarks/expA_async/shaders/mesh_deform.comp:25-34),
//                    with the reproducible sin of rq_device.cuh.
#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;

struct Cam {
    float cx, cy, cz, lx, ly, lz;
};

__global__ void __launch_bounds__(kT) k_gen_procedural(Cam c, uint32_t count, uint32_t coherent,
                                                       rq_ray* __restrict__ rays) {
    const uint32_t idx = blockIdx.x * kT + threadIdx.x;
    if (idx >= count) return;
    rq::F3 o, d;
    if (coherent) {
        rq::F3 cp{c.cx, c.cy, c.cz};
        rq::F3 fwd = rq::f3norm(rq::f3sub(rq::F3{c.lx, c.ly, c.lz}, cp));
        rq::F3 right = rq::f3norm(rq::f3cross(fwd, rq::F3{0.0f, 1.0f, 0.0f}));
        rq::F3 up = rq::f3cross(right, fwd);
        const uint32_t width = 1024, height = (count + width - 1) / width;
        const uint32_t x = idx % width, y = idx / width;
        float u = ((__uint2float_rn(x) + 0.5f) / __uint2float_rn(width)) * 2.0f - 1.0f;
        float v = ((__uint2float_rn(y) + 0.5f) / __uint2float_rn(height)) * 2.0f - 1.0f;
        rq::F3 a{(right.x * u) * 0.55f, (right.y * u) * 0.55f, (right.z * u) * 0.55f};
        rq::F3 b{(up.x * v) * 0.55f, (up.y * v) * 0.55f, (up.z * v) * 0.55f};
        o = cp;
        d = rq::f3norm(rq::F3{(fwd.x + a.x) + b.x, (fwd.y + a.y) + b.y, (fwd.z + a.z) + b.z});
    } else {
        float rx = rq::hash_float(idx * 6 + 0) * 80.0f - 40.0f;
        float ry = rq::hash_float(idx * 6 + 1) * 15.0f + 15.0f;
        float rz = rq::hash_float(idx * 6 + 2) * 80.0f - 40.0f;
        o = {rx, ry, rz};
        float dx = rq::hash_float(idx * 6 + 3) * 0.8f - 0.4f;
        float dy = -1.0f - rq::hash_float(idx * 6 + 4) * 0.5f;
        float dz = rq::hash_float(idx * 6 + 5) * 0.8f - 0.4f;
        d = rq::f3norm(rq::F3{dx, dy, dz});
    }
    float4* out = reinterpret_cast<float4*>(rays + idx);
    out[0] = make_float4(o.x, o.y, o.z, 0.01f);
    out[1] = make_float4(d.x, d.y, d.z, 1000.0f);
}

__global__ void __launch_bounds__(kT) k_deform_wave(const float* __restrict__ base, float* __restrict__ out,
                                                    uint32_t nv, float t, float amp, float freq) {
    const uint32_t v = blockIdx.x * kT + threadIdx.x;
    if (v >= nv) return;
    float x = base[3 * size_t(v)], y = base[3 * size_t(v) + 1], z = base[3 * size_t(v) + 2];
    float s, c;
    rq::sincos_taylor(t + freq * x, &s, &c);
    out[3 * size_t(v)] = x;
    out[3 * size_t(v) + 1] = y;
    out[3 * size_t(v) + 2] = z + amp * s;
}

// Same deformation with the time in device memory: state[0] = t (float
// bits), state[1] = block ticket.  Every block reads t first; the last block
// to take a ticket advances t by dt and clears the ticket, so a captured
// graph moves the mesh forward on every replay.
__global__ void __launch_bounds__(kT) k_deform_wave_step(const float* __restrict__ base, float* __restrict__ out,
                                                         uint32_t nv, uint32_t* state, float dt, float amp,
                                                         float freq) {
    __shared__ float s_t;
    __shared__ bool s_last;
    if (threadIdx.x == 0) s_t = __uint_as_float(rq::ld_acquire(state));
    __syncthreads();
    const float t = s_t;
    const uint32_t v = blockIdx.x * kT + threadIdx.x;
    if (v < nv) {
        const float x = base[3 * size_t(v)], y = base[3 * size_t(v) + 1], z = base[3 * size_t(v) + 2];
        float s, c;
        rq::sincos_taylor(t + freq * x, &s, &c);
        out[3 * size_t(v)] = x;
        out[3 * size_t(v) + 1] = y;
        out[3 * size_t(v) + 2] = z + amp * s;
    }
    if (threadIdx.x == 0) s_last = atomicAdd(state + 1, 1u) == gridDim.x - 1;
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        state[1] = 0u;
        rq::st_release(state, __float_as_uint(t + dt));
    }
}

}  // namespace

int rq_launch_deform_step(rq_ctx* ctx, const float* base, float* out, uint32_t nv, uint32_t* state, float dt,
                          float amp, float freq, cudaStream_t st) {
    if (nv == 0) return RQ_OK;
    k_deform_wave_step<<<(nv + kT - 1) / kT, kT, 0, st>>>(base, out, nv, state, dt, amp, freq);
    return rq_cuda_status(ctx, cudaGetLastError(), "deform step launch");
}

int rq_launch_gen_procedural(rq_ctx* ctx, const float cam[3], const float look[3], uint32_t count,
                             uint32_t coherent, rq_ray* rays, cudaStream_t st) {
    if (count == 0) return RQ_OK;
    Cam c{cam[0], cam[1], cam[2], look[0], look[1], look[2]};
    k_gen_procedural<<<(count + kT - 1) / kT, kT, 0, st>>>(c, count, coherent, rays);
    return rq_cuda_status(ctx, cudaGetLastError(), "procedural ray launch");
}

int rq_launch_deform(rq_ctx* ctx, const float* base, float* out, uint32_t nv, float t, float amp, float freq,
                     cudaStream_t st) {
    if (nv == 0) return RQ_OK;
    k_deform_wave<<<(nv + kT - 1) / kT, kT, 0, st>>>(base, out, nv, t, amp, freq);
    return rq_cuda_status(ctx, cudaGetLastError(), "deform launch");
}

// ------------------------------------------------------------ wait check
namespace {

// One bounded wait on *flag changing from 0: the wait of the grid barriers
// (rq::wait_change), for checking that a wait that runs out reports.
__global__ void k_wait_check(const uint32_t* flag, uint32_t limit, uint32_t* err) {
    if (blockIdx.x == 0 && threadIdx.x == 0) rq::wait_change(flag, 0u, limit, err, RQ_DERR_WAIT_CHECK);
}

}  // namespace

int rq_launch_wait_check(rq_ctx* ctx, const uint32_t* flag, uint32_t limit, cudaStream_t st) {
    k_wait_check<<<1, 32, 0, st>>>(flag, limit, ctx->d_err);
    return rq_cuda_status(ctx, cudaGetLastError(), "wait check launch");
}
