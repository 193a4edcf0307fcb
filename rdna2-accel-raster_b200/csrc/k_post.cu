// k_post.cu — the consumers of the frame's AO on the device.
//
//  k_gbuffer_depth  G-buffer position -> depth z/w of the view-projection
//                   (Vulkan [0,1]; 1.0 where the pixel saw no geometry, as a
//                   cleared depth buffer holds).
//  k_blur_ao        one pass of the depth-aware separable blur of
//                   shaders/bilateral_blur.comp:15-55: a 9-tap Gaussian
//                   (0.227027 centre, 0.1945946, 0.1216216, 0.054054,
//                   0.016216) along one axis, a tap counting only where its
//                   depth is within the threshold of the centre's, centre
//                   pixels at depth >= 1 passed through.  The shader samples
//                   at texel centres (uv = (p + 0.5) / res, offsets of whole
//                   texels), so taps read texels directly, clamped to the edge.
// Operations in the shader's order, one rounding each.
#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

struct Mat4 {
    float m[16];  // column-major
};

__global__ void __launch_bounds__(256) k_gbuffer_depth(const rq_gbuffer_px* __restrict__ gbuf, uint32_t npix,
                                                       const __grid_constant__ Mat4 vp, float* __restrict__ depth) {
    const uint32_t p = blockIdx.x * 256u + threadIdx.x;
    if (p >= npix) return;
    const float4 g = reinterpret_cast<const float4*>(gbuf + p)[0];
    if (__float_as_uint(g.w) == 0u) {
        depth[p] = 1.0f;
        return;
    }
    const float* m = vp.m;
    const float z = ((m[2] * g.x + m[6] * g.y) + m[10] * g.z) + m[14];
    const float w = ((m[3] * g.x + m[7] * g.y) + m[11] * g.z) + m[15];
    depth[p] = z / w;
}

__global__ void __launch_bounds__(256) k_blur_ao(const float* __restrict__ in, const float* __restrict__ depth,
                                                 float* __restrict__ out, uint32_t w, uint32_t h, int dx, int dy,
                                                 float threshold) {
    const uint32_t x = blockIdx.x * 16u + (threadIdx.x & 15u);
    const uint32_t y = blockIdx.y * 16u + (threadIdx.x >> 4);
    if (x >= w || y >= h) return;
    const uint32_t p = y * w + x;
    const float cv = __ldg(in + p), cd = __ldg(depth + p);
    if (cd >= 1.0f) {
        out[p] = cv;
        return;
    }
    const float wt[4] = {0.1945946f, 0.1216216f, 0.054054f, 0.016216f};
    float total = 0.227027f;
    float result = cv * total;
#pragma unroll
    for (int i = 1; i <= 4; ++i) {
        const int px = min(max(int(x) + dx * i, 0), int(w) - 1), py = min(max(int(y) + dy * i, 0), int(h) - 1);
        const int nx = min(max(int(x) - dx * i, 0), int(w) - 1), ny = min(max(int(y) - dy * i, 0), int(h) - 1);
        const uint32_t qp = uint32_t(py) * w + uint32_t(px), qn = uint32_t(ny) * w + uint32_t(nx);
        const float wp = wt[i - 1] * (fabsf(__ldg(depth + qp) - cd) < threshold ? 1.0f : 0.0f);
        result = result + __ldg(in + qp) * wp;
        total = total + wp;
        const float wn = wt[i - 1] * (fabsf(__ldg(depth + qn) - cd) < threshold ? 1.0f : 0.0f);
        result = result + __ldg(in + qn) * wn;
        total = total + wn;
    }
    out[p] = result / fmaxf(total, 0.001f);
}

}  // namespace

int rq_launch_gbuffer_depth(rq_ctx* ctx, const rq_gbuffer_px* gbuf, uint32_t npix, const float vp[16], float* depth,
                            cudaStream_t st) {
    if (npix == 0) return RQ_OK;
    Mat4 m;
    for (int i = 0; i < 16; ++i) m.m[i] = vp[i];
    k_gbuffer_depth<<<(npix + 255) / 256, 256, 0, st>>>(gbuf, npix, m, depth);
    return rq_cuda_status(ctx, cudaGetLastError(), "gbuffer depth launch");
}

int rq_launch_blur_ao(rq_ctx* ctx, const float* in, const float* depth, float* out, uint32_t w, uint32_t h, int dx,
                      int dy, float threshold, cudaStream_t st) {
    if (w == 0 || h == 0) return RQ_OK;
    dim3 grid((w + 15) / 16, (h + 15) / 16);
    k_blur_ao<<<grid, 256, 0, st>>>(in, depth, out, w, h, dx, dy, threshold);
    return rq_cuda_status(ctx, cudaGetLastError(), "ao blur launch");
}
