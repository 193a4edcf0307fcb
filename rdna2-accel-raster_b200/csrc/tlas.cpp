// tlas.cpp — C ABI of two-level scenes (include/rq.h): the instance table
// (inverse transforms in double precision, rounded once), the instance boxes
// and the top-level LBVH over them, and the two-level traversal launch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

#include "rq_tlas.h"

namespace {

// Inverse of the affine map x -> A x + t (A row-major 3x3, t the last
// column): A^-1 = adj(A) / det(A), translation -A^-1 t; double precision,
// each entry rounded to float once.  Returns false for a singular A.
bool affine_inverse(const float* f, float* inv) {
    const double a[3][3] = {{f[0], f[1], f[2]}, {f[4], f[5], f[6]}, {f[8], f[9], f[10]}};
    const double t[3] = {f[3], f[7], f[11]};
    const double c00 = a[1][1] * a[2][2] - a[1][2] * a[2][1];
    const double c01 = a[1][2] * a[2][0] - a[1][0] * a[2][2];
    const double c02 = a[1][0] * a[2][1] - a[1][1] * a[2][0];
    const double det = a[0][0] * c00 + a[0][1] * c01 + a[0][2] * c02;
    if (!(std::fabs(det) > 0.0) || !std::isfinite(det)) return false;
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
        for (int c = 0; c < 3; ++c) inv[4 * r + c] = float(m[r][c]);
        inv[4 * r + 3] = float(tr);
    }
    return true;
}

void free_tlas(rq_tlas* t) {
    if (t->top) rq_bvh_destroy(t->top);
    if (t->d_inst) cudaFree(t->d_inst);
    if (t->d_fwd) cudaFree(t->d_fwd);
    if (t->d_tri9) cudaFree(t->d_tri9);
    delete t;
}

}  // namespace

extern "C" {

int rq_tlas_build(rq_ctx* ctx, const rq_instance* instances, uint32_t n, rq_tlas** out, rq_stream stream) {
    if (!ctx || !instances || !out || n == 0) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "bad instance list");
    if (n >= RQ_MAX_TRIANGLES) return rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "too many instances");
    cudaSetDevice(ctx->device);
    std::vector<TlasInst> inst(n);
    std::vector<float> fwd(12ull * n);
    uint32_t blas_bound = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const rq_instance& s = instances[i];
        if (!s.blas) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "instance without a BLAS");
        rq_bvh_info inf{};
        int rc = rq_bvh_info_get(const_cast<rq_bvh*>(s.blas), &inf);
        if (rc) return rc;
        if (!s.blas->has4 || s.blas->device != ctx->device)
            return rq_set_error(ctx, RQ_ERR_STATE, "instance BLAS has no 4-wide BVH on this device");
        for (int k = 0; k < 12; ++k)
            if (!std::isfinite(s.transform[k])) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "non-finite transform");
        if (!affine_inverse(s.transform, inst[i].inv))
            return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "singular instance transform");
        std::copy(s.transform, s.transform + 12, fwd.begin() + 12ull * i);
        inst[i].nodes = s.blas->nodes4;
        inst[i].tris = s.blas->tris;
        inst[i].perm = s.blas->perm;
        inst[i].instance_id = s.instance_id;
        inst[i].mask = s.mask;
        blas_bound = std::max(blas_bound, 3u * (inf.depth4 + 2u) + 1u);
    }
    rq_tlas* t = new (std::nothrow) rq_tlas();
    if (!t) return RQ_ERR_OOM;
    t->ctx = ctx;
    t->device = ctx->device;
    t->num_instances = n;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMalloc(&t->d_inst, sizeof(TlasInst) * n);
    if (e == cudaSuccess) e = cudaMalloc(&t->d_fwd, sizeof(float) * 12ull * n);
    if (e == cudaSuccess) e = cudaMalloc(&t->d_tri9, sizeof(float) * 9ull * n);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_inst, inst.data(), sizeof(TlasInst) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->d_fwd, fwd.data(), sizeof(float) * 12ull * n, cudaMemcpyHostToDevice);
    int rc = e == cudaSuccess ? RQ_OK : rq_cuda_status(ctx, e, "instance table");
    if (rc == RQ_OK) rc = rq_launch_instance_boxes(ctx, t->d_inst, t->d_fwd, n, t->d_tri9, st);
    if (rc == RQ_OK) rc = rq_build(ctx, t->d_tri9, 12, 3 * n, nullptr, n, 1, RQ_BUILD_BVH4, &t->top, stream);
    rq_bvh_info top{};
    if (rc == RQ_OK) rc = rq_bvh_info_get(t->top, &top);
    if (rc == RQ_OK) {
        t->stack_bound = 3u * (top.depth4 + 2u) + 1u + 1u + blas_bound;
        if (t->stack_bound > 256u) rc = rq_set_error(ctx, RQ_ERR_UNSUPPORTED, "scene too deep for the stack");
    }
    if (rc) {
        free_tlas(t);
        return rc;
    }
    t->last_stream = st;
    *out = t;
    return RQ_OK;
}

int rq_tlas_trace(rq_ctx* ctx, const rq_tlas* tlas, const rq_ray* rays, uint32_t n, uint32_t flags,
                  uint32_t cull_mask, rq_hit* hits, rq_stream stream) {
    if (!ctx || !tlas || (n && (!rays || !hits))) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "null argument");
    if (flags & ~3u) return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "unknown trace flags");
    if ((reinterpret_cast<uintptr_t>(rays) | reinterpret_cast<uintptr_t>(hits)) & 15u)
        return rq_set_error(ctx, RQ_ERR_INVALID_ARG, "misaligned ray/hit buffer");
    cudaSetDevice(ctx->device);
    return rq_launch_trace_tlas(ctx, tlas, rays, n, flags, cull_mask, hits, static_cast<cudaStream_t>(stream));
}

int rq_tlas_destroy(rq_tlas* tlas) {
    if (!tlas) return RQ_ERR_INVALID_ARG;
    cudaSetDevice(tlas->device);
    if (tlas->last_stream) cudaStreamSynchronize(tlas->last_stream);
    free_tlas(tlas);
    return RQ_OK;
}

}  // extern "C"
