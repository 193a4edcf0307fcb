// k_radv.cu — the RADV image of shaders/fast_bvh_builder.comp:91-257 for any
// triangle count, in one launch.
//
// The image is an implicit 4-ary tree over the triangles in input order
// (level plan of include/radv_bvh.hpp:193-215): 64-B triangle nodes, Box32
// leaves over four consecutive triangles, parents over four consecutive
// children, qNaN boxes with child 0xFFFFFFFF in empty slots, the 136-B header
// and the pre-root dwords at bytes 180 (= 5) and 188 (= 0xFFFFFFFF).  Bytes
// the shader never writes (136..191 apart from those two dwords) are zeroed.
//
// Block b owns leaf boxes [1024b, 1024b+1024): 4096 triangles, one per
// thread per round, so the four triangles of a leaf box sit in four
// consecutive lanes and their boxes meet through warp shuffles.  The block
// then reduces its subtree in shared memory for up to five levels.  The last
// block to finish (atomic ticket) builds the remaining top levels and the
// header from the per-block subtree boxes.
#include <algorithm>
#include <mutex>

#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;
constexpr int kLeafBoxes = 1024;  // per block
constexpr uint32_t kQNaN = 0x7fc00000u;

struct RadvArgs {
    const float* tri9;
    uint32_t n;
    uint8_t* img;
    uint32_t levels;
    uint32_t total_boxes;
    uint32_t counts[16];
    uint32_t offs[16];
    float4* top;        // 2 per block: subtree box lo, hi (then reused for the top levels)
    uint32_t* ticket;
    uint64_t size;
    uint32_t check_header = 0;  // refit: the image's header must already describe n triangles
    uint32_t* err = nullptr;
};

__device__ __forceinline__ void write_box(uint8_t* boxes, uint32_t node, const uint32_t ch[4], const float mn[4][3],
                                          const float mx[4][3]) {
    float4* o = reinterpret_cast<float4*>(boxes + 128ull * node);
    float c[24];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        c[6 * k + 0] = mn[k][0];
        c[6 * k + 1] = mn[k][1];
        c[6 * k + 2] = mn[k][2];
        c[6 * k + 3] = mx[k][0];
        c[6 * k + 4] = mx[k][1];
        c[6 * k + 5] = mx[k][2];
    }
    reinterpret_cast<uint4*>(o)[0] = make_uint4(ch[0], ch[1], ch[2], ch[3]);
#pragma unroll
    for (int q = 0; q < 6; ++q) o[1 + q] = make_float4(c[4 * q], c[4 * q + 1], c[4 * q + 2], c[4 * q + 3]);
    reinterpret_cast<uint4*>(o)[7] = make_uint4(0u, 0u, 0u, 0u);
}

// Parent box over up to four children held in (cmn, cmx); writes the Box32
// node and returns the union through (umn, umx).
__device__ __forceinline__ void make_parent(uint8_t* boxes, uint32_t node, uint32_t child_global0, uint32_t nvalid,
                                            const float* cmn, const float* cmx, float umn[3], float umx[3]) {
    uint32_t ch[4];
    float mn[4][3], mx[4][3];
    const float qn = __uint_as_float(kQNaN);
    umn[0] = umn[1] = umn[2] = 1e30f;
    umx[0] = umx[1] = umx[2] = -1e30f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (uint32_t(c) < nvalid) {
            ch[c] = (((child_global0 + c) * 128u) >> 3) | RQ_RADV_NODE_BOX32;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn[c][k] = cmn[3 * c + k];
                mx[c][k] = cmx[3 * c + k];
                umn[k] = fminf(umn[k], mn[c][k]);
                umx[k] = fmaxf(umx[k], mx[c][k]);
            }
        } else {
            ch[c] = RQ_RADV_INVALID_NODE;
#pragma unroll
            for (int k = 0; k < 3; ++k) mn[c][k] = mx[c][k] = qn;
        }
    }
    write_box(boxes, node, ch, mn, mx);
}

__device__ void write_header(const RadvArgs& A, const float mn[3], const float mx[3]) {
    uint32_t* h = reinterpret_cast<uint32_t*>(A.img);
    // zero 0..191, then fill the fields
    for (int i = 0; i < 48; ++i) h[i] = 0u;
    h[0] = 192u;  // bvh_offset
    h[1] = 0u;    // root_flags
    for (int k = 0; k < 3; ++k) {
        h[2 + k] = __float_as_uint(mn[k]);
        h[5 + k] = __float_as_uint(mx[k]);
    }
    h[8] = 8u;  // update_dispatch_size
    h[9] = 1u;
    h[10] = 1u;
    uint64_t* h64 = reinterpret_cast<uint64_t*>(A.img);
    h64[0x30 / 8] = A.size;        // compacted_size
    h64[0x38 / 8] = A.size + 128;  // serialization_size
    h[0x40 / 4] = 1u;              // copy_dispatch_size
    h[0x44 / 4] = 1u;
    h[0x48 / 4] = 1u;
    h64[0x50 / 8] = A.size;  // size
    h[0x58 / 4] = 0u;        // geometry_type
    h[0x5C / 4] = 1u;        // geometry_count
    h64[0x60 / 8] = 192ull + 128ull * A.total_boxes;  // leaf_nodes_offset
    h64[0x68 / 8] = A.n;                              // primitive_count
    h64[0x70 / 8] = 0ull;                             // instance_count
    h[0x78 / 4] = 0u;                                 // leaf_node_offsets_offset
    h[0x7C / 4] = 4u;                                 // build_flags
    h[0x80 / 4] = 1u;                                 // type
    h[180 / 4] = 5u;
    h[188 / 4] = 0xffffffffu;
}

__global__ void __launch_bounds__(kT) k_radv(RadvArgs A) {
    // leaf-level boxes (1024) and the first parent level (256) ping-pong
    __shared__ float s_mn0[kLeafBoxes * 3], s_mx0[kLeafBoxes * 3];
    __shared__ float s_mn1[kLeafBoxes / 4 * 3], s_mx1[kLeafBoxes / 4 * 3];
    __shared__ uint32_t s_last;
    float* cmn_src = s_mn0;
    float* cmx_src = s_mx0;
    float* cmn_dst = s_mn1;
    float* cmx_dst = s_mx1;
    if (A.check_header && blockIdx.x == 0 && threadIdx.x == 0) {
        // read before this block takes its ticket, so before the last block
        // rewrites the header
        const uint32_t* h = reinterpret_cast<const uint32_t*>(A.img);
        const uint64_t* h64 = reinterpret_cast<const uint64_t*>(A.img);
        if (h[0] != 192u || h64[0x60 / 8] != 192ull + 128ull * A.total_boxes || h64[0x68 / 8] != A.n ||
            h64[0x50 / 8] != A.size)
            rq::set_err(A.err, RQ_DERR_RADV_IMAGE);
    }
    const uint32_t L = A.levels;
    const uint32_t leaf_lvl = L - 1;
    const uint32_t leaf_cnt = A.counts[leaf_lvl];
    uint8_t* boxes = A.img + 192;
    uint8_t* trin = A.img + 192 + 128ull * A.total_boxes;
    const uint32_t lane = threadIdx.x & 31;
    const float qn = __uint_as_float(kQNaN);

    // ---- leaf boxes and triangle nodes
    const uint32_t lb0 = blockIdx.x * kLeafBoxes;
    const uint32_t nlb = min(uint32_t(kLeafBoxes), leaf_cnt - lb0);
    // rounds of kT triangles that hold any of this block's (fewer than 16
    // for a small image; the same for every thread)
    const uint32_t rounds = (nlb * 4u + kT - 1) / kT;
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t local = r * kT + threadIdx.x;  // triangle within block
        const uint32_t ti = lb0 * 4u + local;
        const bool valid = local < nlb * 4u && ti < A.n;
        float tmn[3] = {qn, qn, qn}, tmx[3] = {qn, qn, qn};
        if (valid) {
            const float* v = A.tri9 + 9ull * ti;
            float f[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) f[q] = __ldg(v + q);
            float4* o = reinterpret_cast<float4*>(trin + 64ull * ti);
            o[0] = make_float4(f[0], f[1], f[2], f[3]);
            o[1] = make_float4(f[4], f[5], f[6], f[7]);
            o[2] = make_float4(f[8], 0.0f, 0.0f, 0.0f);
            reinterpret_cast<uint4*>(o)[3] =
                make_uint4(ti, RQ_RADV_GEOMETRY_OPAQUE, 0u, RQ_RADV_BARYCENTRICS_CONTROL_DEFAULT);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                tmn[k] = fminf(f[k], fminf(f[3 + k], f[6 + k]));
                tmx[k] = fmaxf(f[k], fmaxf(f[3 + k], f[6 + k]));
            }
        }
        // gather the four triangles of this lane's leaf box (lanes 4j..4j+3)
        const uint32_t g0 = lane & ~3u;
        uint32_t okm = __ballot_sync(0xffffffffu, valid);
        float cmn[4][3], cmx[4][3];
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cmn[c][k] = __shfl_sync(0xffffffffu, tmn[k], g0 + c);
                cmx[c][k] = __shfl_sync(0xffffffffu, tmx[k], g0 + c);
            }
        const uint32_t lbl = local >> 2;  // leaf box within block
        if ((lane & 3u) == 0u && lbl < nlb) {
            uint32_t ch[4];
            float umn[3] = {1e30f, 1e30f, 1e30f}, umx[3] = {-1e30f, -1e30f, -1e30f};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                if ((okm >> (g0 + c)) & 1u) {
                    uint32_t tic = (lb0 + lbl) * 4u + c;
                    ch[c] = ((A.total_boxes * 128u + tic * 64u) >> 3) | RQ_RADV_NODE_TRIANGLE;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        umn[k] = fminf(umn[k], cmn[c][k]);
                        umx[k] = fmaxf(umx[k], cmx[c][k]);
                    }
                } else {
                    ch[c] = RQ_RADV_INVALID_NODE;
#pragma unroll
                    for (int k = 0; k < 3; ++k) cmn[c][k] = cmx[c][k] = qn;
                }
            }
            write_box(boxes, A.offs[leaf_lvl] + lb0 + lbl, ch, cmn, cmx);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                s_mn0[3 * lbl + k] = umn[k];
                s_mx0[3 * lbl + k] = umx[k];
            }
        }
    }
    __syncthreads();

    // ---- in-block levels (up to five)
    uint32_t nchild = nlb;                // children at the current level in this block
    uint32_t child_base = lb0;            // first child index within its level
    uint32_t lvl = leaf_lvl;              // level of the children
    for (uint32_t j = 1; j <= 5 && lvl > 0; ++j) {
        const uint32_t plvl = lvl - 1;
        const uint32_t np = (nchild + 3) / 4;
        const uint32_t pbase = child_base >> 2;
        for (uint32_t t = threadIdx.x; t < np; t += kT) {
            uint32_t nv = min(4u, nchild - 4 * t);
            float umn[3], umx[3];
            make_parent(boxes, A.offs[plvl] + pbase + t, A.offs[lvl] + child_base + 4 * t, nv, cmn_src + 12 * t,
                        cmx_src + 12 * t, umn, umx);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cmn_dst[3 * t + k] = umn[k];
                cmx_dst[3 * t + k] = umx[k];
            }
        }
        __syncthreads();
        float* tn = cmn_src;
        cmn_src = cmn_dst;
        cmn_dst = tn;
        float* tx = cmx_src;
        cmx_src = cmx_dst;
        cmx_dst = tx;
        nchild = np;
        child_base = pbase;
        lvl = plvl;
    }

    if (lvl == 0) {
        // this block built the root (single-block image)
        if (threadIdx.x == 0) {
            float mn[3] = {cmn_src[0], cmn_src[1], cmn_src[2]};
            float mx[3] = {cmx_src[0], cmx_src[1], cmx_src[2]};
            write_header(A, mn, mx);
        }
        return;
    }

    // ---- publish the subtree box, last block finishes the top
    if (threadIdx.x == 0) {
        __stcg(A.top + 2 * blockIdx.x, make_float4(cmn_src[0], cmn_src[1], cmn_src[2], 0.0f));
        __stcg(A.top + 2 * blockIdx.x + 1, make_float4(cmx_src[0], cmx_src[1], cmx_src[2], 0.0f));
        __threadfence();
        s_last = atomicAdd(A.ticket, 1u) == gridDim.x - 1 ? 1u : 0u;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // level `lvl` holds gridDim.x nodes whose boxes are in A.top[2b], A.top[2b+1]
    float4* src = A.top;
    float4* dst = A.top + 2 * gridDim.x;
    uint32_t ncnt = A.counts[lvl];
    while (lvl > 0) {
        const uint32_t plvl = lvl - 1;
        const uint32_t np = A.counts[plvl];
        for (uint32_t t = threadIdx.x; t < np; t += kT) {
            uint32_t nv = min(4u, ncnt - 4 * t);
            float cmn[12], cmx[12];
            for (uint32_t c = 0; c < nv; ++c) {
                float4 a = __ldcg(src + 2 * (4 * t + c)), b = __ldcg(src + 2 * (4 * t + c) + 1);
                cmn[3 * c] = a.x;
                cmn[3 * c + 1] = a.y;
                cmn[3 * c + 2] = a.z;
                cmx[3 * c] = b.x;
                cmx[3 * c + 1] = b.y;
                cmx[3 * c + 2] = b.z;
            }
            float umn[3], umx[3];
            make_parent(boxes, A.offs[plvl] + t, A.offs[lvl] + 4 * t, nv, cmn, cmx, umn, umx);
            __stcg(dst + 2 * t, make_float4(umn[0], umn[1], umn[2], 0.0f));
            __stcg(dst + 2 * t + 1, make_float4(umx[0], umx[1], umx[2], 0.0f));
        }
        __threadfence();
        __syncthreads();
        float4* tmp = src;
        src = dst;
        dst = tmp;
        ncnt = np;
        lvl = plvl;
    }
    if (threadIdx.x == 0) {
        float4 a = __ldcg(src), b = __ldcg(src + 1);
        float mn[3] = {a.x, a.y, a.z}, mx[3] = {b.x, b.y, b.z};
        write_header(A, mn, mx);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Allocation-free RADV build.  Some callers own every byte of device memory
// they use — they size their buffers up front from their own pool or budget
// and cannot let a library call cudaMalloc / cudaFree, which synchronise the
// whole device and can fail mid-frame.  This variant takes only the vertex
// buffer and the image buffer from the caller; its scratch (the finishing
// ticket and two boxes per block for the top levels) lives in the static
// device array below, sized for at most RQ_RADV_NOALLOC_MAX_TRIANGLES
// triangles.  Every GPU that loads librq.so holds the array until the
// process exits.
static __device__ __align__(256) unsigned char rq_radv_noalloc_scratch
    [256 + 4 * sizeof(float4) * ((RQ_RADV_NOALLOC_MAX_TRIANGLES / 4 + kLeafBoxes - 1) / kLeafBoxes)];

namespace {
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[256] = {};  // device address of the array, per device ordinal
}  // namespace

extern "C" int rq_build_radv_noalloc(const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                                     rq_stream stream) {
    if (!tri9 || !as_image || num_triangles == 0) return RQ_ERR_INVALID_ARG;
    if (num_triangles > RQ_RADV_NOALLOC_MAX_TRIANGLES) return RQ_ERR_UNSUPPORTED;
    if (reinterpret_cast<uintptr_t>(as_image) & 15u) return RQ_ERR_INVALID_ARG;
    rq_radv_layout L;
    if (rq_radv_layout_get(num_triangles, &L) != RQ_OK) return RQ_ERR_UNSUPPORTED;
    if (as_bytes < L.total_as_size) return RQ_ERR_SIZE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return RQ_ERR_NO_DEVICE;
    void* base = nullptr;
    {
        // set-up once per device, with that device current: the host-side
        // name of the array is not a device address
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, rq_radv_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return RQ_ERR_CUDA;
            }
            g_noalloc_ptr[dev] = p;
        }
        base = g_noalloc_ptr[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RadvArgs a;
    a.tri9 = tri9;
    a.n = num_triangles;
    a.img = static_cast<uint8_t*>(as_image);
    a.levels = L.num_levels;
    a.total_boxes = L.total_boxes;
    for (int i = 0; i < 16; ++i) {
        a.counts[i] = L.level_counts[i];
        a.offs[i] = L.level_offsets[i];
    }
    a.ticket = static_cast<uint32_t*>(base);
    a.top = reinterpret_cast<float4*>(static_cast<char*>(base) + 256);
    a.size = L.total_as_size;
    // the array keeps the previous call's contents: the ticket must start at 0
    if (cudaMemsetAsync(a.ticket, 0, sizeof(uint32_t), st) != cudaSuccess) {
        cudaGetLastError();
        return RQ_ERR_CUDA;
    }
    const uint32_t leaf_cnt = L.level_counts[L.num_levels - 1];
    k_radv<<<(leaf_cnt + kLeafBoxes - 1) / kLeafBoxes, kT, 0, st>>>(a);
    if (cudaGetLastError() != cudaSuccess) return RQ_ERR_CUDA;
    return RQ_OK;
}

int rq_launch_radv(rq_ctx* ctx, const float* tri9, uint32_t n, void* img, const rq_radv_layout& L, cudaStream_t st,
                   bool refit) {
    const uint32_t leaf_cnt = L.level_counts[L.num_levels - 1];
    const uint32_t blocks = (leaf_cnt + kLeafBoxes - 1) / kLeafBoxes;
    size_t need = sizeof(float4) * 4ull * blocks + 256;
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    RadvArgs a;
    a.tri9 = tri9;
    a.n = n;
    a.img = static_cast<uint8_t*>(img);
    a.levels = L.num_levels;
    a.total_boxes = L.total_boxes;
    for (int i = 0; i < 16; ++i) {
        a.counts[i] = L.level_counts[i];
        a.offs[i] = L.level_offsets[i];
    }
    a.ticket = static_cast<uint32_t*>(ctx->scratch);
    a.top = reinterpret_cast<float4*>(static_cast<char*>(ctx->scratch) + 256);
    a.size = L.total_as_size;
    a.check_header = refit ? 1u : 0u;
    a.err = ctx->d_err;
    if (blocks > 1) cudaMemsetAsync(a.ticket, 0, sizeof(uint32_t), st);  // one block never takes a ticket
    k_radv<<<blocks, kT, 0, st>>>(a);
    return rq_cuda_status(ctx, cudaGetLastError(), "radv build launch");
}

// ------------------------------------------------------------ validation
// Decode a whole RADV image on the device and check its invariants.  Box
// nodes sit at 128-B strides from the root up to the leaf region, triangle
// nodes at 64-B strides after it (the header says where).  One thread per
// box node checks its four children:
//  - the child id decodes to an offset inside the right region and stride
//    (every read below is range-checked first, so a corrupt image is only
//    counted, never dereferenced out of bounds);
//  - a Box32 child's box equals the union of that node's child boxes, a
//    triangle child's box equals its triangle's bounds;
//  - references per node and per triangle id are counted.
// A second pass counts nodes referenced other than exactly once (the root:
// never) and triangle ids not seen exactly once.
namespace {

struct RadvCheckArgs {
    const uint8_t* img;
    uint64_t bytes;
    uint32_t root;
    uint64_t leaf_off;
    uint32_t boxes;
    uint32_t tris;
    uint32_t* box_refs;  // boxes
    uint32_t* tri_refs;  // tris
    uint32_t* id_refs;   // tris
    unsigned long long* out;  // rq_radv_check counters
};

__device__ __forceinline__ void box_of(const rq_radv_box32& b, float mn[3], float mx[3], uint32_t& valid) {
    valid = 0;
    for (int k = 0; k < 3; ++k) {
        mn[k] = INFINITY;
        mx[k] = -INFINITY;
    }
    for (int c = 0; c < 4; ++c) {
        if (b.children[c] == RQ_RADV_INVALID_NODE) continue;
        ++valid;
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], b.coords[c][k]);
            mx[k] = fmaxf(mx[k], b.coords[c][3 + k]);
        }
    }
}

__global__ void __launch_bounds__(256) k_radv_check(RadvCheckArgs a) {
    const uint32_t b = blockIdx.x * 256u + threadIdx.x;
    if (b >= a.boxes) return;
    unsigned long long bad_off = 0, bad_box = 0, tri_nodes = 0, box_children = 0;
    rq_radv_box32 node;
    memcpy(&node, a.img + a.root + 128ull * b, sizeof(node));
    for (int c = 0; c < 4; ++c) {
        const uint32_t id = node.children[c];
        if (id == RQ_RADV_INVALID_NODE) continue;
        const uint64_t at = uint64_t(a.root) + (uint64_t(id & ~7u) << 3);
        const uint32_t type = id & 7u;
        if (type == RQ_RADV_NODE_BOX32) {
            const uint64_t rel = at - a.root;
            if (at < a.root || rel % 128u || rel / 128u >= a.boxes || at + 128u > a.bytes) {
                ++bad_off;
                continue;
            }
            const uint32_t cb = uint32_t(rel / 128u);
            atomicAdd(a.box_refs + cb, 1u);
            ++box_children;
            rq_radv_box32 child;
            memcpy(&child, a.img + at, sizeof(child));
            float mn[3], mx[3];
            uint32_t valid;
            box_of(child, mn, mx, valid);
            bool same = valid > 0;
            for (int k = 0; k < 3; ++k)
                same = same && mn[k] == node.coords[c][k] && mx[k] == node.coords[c][3 + k];
            if (!same) ++bad_box;
        } else if (type == RQ_RADV_NODE_TRIANGLE) {
            if (at < a.leaf_off || (at - a.leaf_off) % 64u || (at - a.leaf_off) / 64u >= a.tris || at + 64u > a.bytes) {
                ++bad_off;
                continue;
            }
            atomicAdd(a.tri_refs + uint32_t((at - a.leaf_off) / 64u), 1u);
            ++tri_nodes;
            rq_radv_tri t;
            memcpy(&t, a.img + at, sizeof(t));
            if (t.triangle_id < a.tris) atomicAdd(a.id_refs + t.triangle_id, 1u);
            bool same = true;
            for (int k = 0; k < 3; ++k) {
                const float lo = fminf(fminf(t.coords[0][k], t.coords[1][k]), t.coords[2][k]);
                const float hi = fmaxf(fmaxf(t.coords[0][k], t.coords[1][k]), t.coords[2][k]);
                same = same && lo == node.coords[c][k] && hi == node.coords[c][3 + k];
            }
            if (!same) ++bad_box;
        } else {
            ++bad_off;
        }
    }
    if (bad_off) atomicAdd(a.out + 2, bad_off);
    if (bad_box) atomicAdd(a.out + 3, bad_box);
    if (tri_nodes) atomicAdd(a.out + 1, tri_nodes);
    if (box_children) atomicAdd(a.out + 0, box_children);
}

__global__ void __launch_bounds__(256) k_radv_check_refs(RadvCheckArgs a) {
    const uint32_t i = blockIdx.x * 256u + threadIdx.x;
    unsigned long long wrong_box = 0, wrong_tri = 0, wrong_id = 0;
    if (i < a.boxes && a.box_refs[i] != (i == 0 ? 0u : 1u)) wrong_box = 1;
    if (i < a.tris && a.tri_refs[i] != 1u) wrong_tri = 1;
    if (i < a.tris && a.id_refs[i] != 1u) wrong_id = 1;
    if (wrong_box) atomicAdd(a.out + 4, wrong_box);
    if (wrong_tri) atomicAdd(a.out + 5, wrong_tri);
    if (wrong_id) atomicAdd(a.out + 6, wrong_id);
}

}  // namespace

int rq_launch_radv_check(rq_ctx* ctx, const void* img, uint64_t bytes, rq_radv_check* out, cudaStream_t st) {
    rq_radv_check r{};
    if (bytes < sizeof(rq_radv_header)) {
        r.header_ok = 0;
        *out = r;
        return RQ_OK;
    }
    rq_radv_header h;
    cudaError_t e = cudaMemcpyAsync(&h, img, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "radv header read");
    const uint64_t n = h.primitive_count;
    r.header_ok = h.bvh_offset >= sizeof(rq_radv_header) && h.leaf_nodes_offset >= h.bvh_offset &&
                  (h.leaf_nodes_offset - h.bvh_offset) % 128u == 0 && n > 0 && n < (1ull << 30) &&
                  h.leaf_nodes_offset + 64ull * n <= bytes && h.size <= bytes;
    if (!r.header_ok) {
        *out = r;
        return RQ_OK;
    }
    const uint32_t boxes = uint32_t((h.leaf_nodes_offset - h.bvh_offset) / 128u);
    r.box_nodes = boxes;
    r.triangle_nodes = n;
    const size_t need = sizeof(unsigned long long) * 8 + sizeof(uint32_t) * (size_t(boxes) + 2 * n) + 256;
    int rc = rq_ensure_scratch(ctx, need, st);
    if (rc) return rc;
    Carve c{reinterpret_cast<uintptr_t>(ctx->scratch), 0};
    RadvCheckArgs a;
    a.img = static_cast<const uint8_t*>(img);
    a.bytes = bytes;
    a.root = h.bvh_offset;
    a.leaf_off = h.leaf_nodes_offset;
    a.boxes = boxes;
    a.tris = uint32_t(n);
    a.out = c.take<unsigned long long>(8);
    a.box_refs = c.take<uint32_t>(boxes);
    a.tri_refs = c.take<uint32_t>(n);
    a.id_refs = c.take<uint32_t>(n);
    e = cudaMemsetAsync(ctx->scratch, 0, c.off, st);
    if (e == cudaSuccess) {
        k_radv_check<<<(boxes + 255) / 256, 256, 0, st>>>(a);
        const uint32_t m = std::max<uint32_t>(boxes, uint32_t(n));
        k_radv_check_refs<<<(m + 255) / 256, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    unsigned long long cnt[8] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, a.out, sizeof(cnt), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return rq_cuda_status(ctx, e, "radv check");
    r.box_children = cnt[0];
    r.triangle_children = cnt[1];
    r.bad_offsets = cnt[2];
    r.bad_boxes = cnt[3];
    r.box_refs_wrong = cnt[4];
    r.triangle_refs_wrong = cnt[5];
    r.ids_wrong = cnt[6];
    *out = r;
    return RQ_OK;
}
