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
// Block b owns leaf boxes [LB*b, LB*b+LB) (LB = 64, 256 or 1024, a power of four):
// 4*LB triangles in rounds of one per thread.  In a multi-block image each
// warp stages its 32 triangles in shared memory so that the triangle and
// leaf box nodes go out as coalesced 16-B stores; a one-block image (up to
// 256 triangles) has each lane read and write its own triangle instead.
// The block then reduces its subtree in shared memory for log4(LB) levels.
// The last block to finish (atomic ticket) builds the remaining top levels
// and the header from the per-block subtree boxes, then puts the ticket back
// to 0 for the next launch on the stream.  Up to 131,072 triangles the
// subtrees are 64 leaf boxes (a 4,096-triangle image is 16 blocks of one
// round), from 4,194,304 on 1024, 256 between.
#include <algorithm>

#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kT = 256;
// 64-leaf-box subtrees up to this many blocks, 256-leaf-box ones above
constexpr uint32_t kSmallBlocksMax = 512;
// 1024-leaf-box subtrees (16 rounds, so the read-ahead of the next round
// covers more of the block's life) from this many blocks on
constexpr uint32_t kLargeBlocksMin = 1024;

// leaf boxes per block (measured on B200): 64 while that gives at most
// kSmallBlocksMax blocks, 1024 from kLargeBlocksMin blocks, 256 between
uint32_t radv_leaf_boxes(uint32_t leaf_cnt) {
    if (leaf_cnt <= 64u * kSmallBlocksMax) return 64u;
    return leaf_cnt >= 1024u * kLargeBlocksMin ? 1024u : 256u;
}
// blocks for a given subtree size
uint32_t radv_blocks(uint32_t leaf_cnt, uint32_t lb) { return (leaf_cnt + lb - 1) / lb; }
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
    uint32_t* ticket;   // 0 at launch; the last block puts it back to 0
    uint64_t size;
    uint32_t check_header = 0;  // refit: the image's header must already describe n triangles
    uint32_t* err = nullptr;
};

// Box32 node over up to four children, child c's bounds fetched by
// get(c, mn, mx); writes the node and returns the union through (umn, umx).
// The union runs over the children in order 0..3, as the shader's min/max
// chain does.
template <class Get>
__device__ __forceinline__ void make_parent(uint8_t* boxes, uint32_t node, uint32_t child_global0, uint32_t nvalid,
                                            Get get, float umn[3], float umx[3]) {
    const float qn = __uint_as_float(kQNaN);
    uint8_t* nd = boxes + 128ull * node;
    uint32_t ch[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
        ch[c] = uint32_t(c) < nvalid ? (((child_global0 + c) * 128u) >> 3) | RQ_RADV_NODE_BOX32 : RQ_RADV_INVALID_NODE;
    reinterpret_cast<uint4*>(nd)[0] = make_uint4(ch[0], ch[1], ch[2], ch[3]);
    umn[0] = umn[1] = umn[2] = 1e30f;
    umx[0] = umx[1] = umx[2] = -1e30f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float mn[3] = {qn, qn, qn}, mx[3] = {qn, qn, qn};
        if (uint32_t(c) < nvalid) {
            get(c, mn, mx);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                umn[k] = fminf(umn[k], mn[k]);
                umx[k] = fmaxf(umx[k], mx[k]);
            }
        }
        float2* b = reinterpret_cast<float2*>(nd + 16 + 24 * c);
        b[0] = make_float2(mn[0], mn[1]);
        b[1] = make_float2(mn[2], mx[0]);
        b[2] = make_float2(mx[1], mx[2]);
    }
    reinterpret_cast<uint4*>(nd)[7] = make_uint4(0u, 0u, 0u, 0u);
}

// children held as 3 floats each in shared memory
struct SmemChildren {
    const float* mn;
    const float* mx;
    __device__ __forceinline__ void operator()(int c, float m[3], float x[3]) const {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            m[k] = mn[3 * c + k];
            x[k] = mx[3 * c + k];
        }
    }
};

// children held as (lo, hi) float4 pairs in global memory (L2)
struct GlobalChildren {
    const float4* p;
    __device__ __forceinline__ void operator()(int c, float m[3], float x[3]) const {
        const float4 a = __ldcg(p + 2 * c), b = __ldcg(p + 2 * c + 1);
        m[0] = a.x;
        m[1] = a.y;
        m[2] = a.z;
        x[0] = b.x;
        x[1] = b.y;
        x[2] = b.z;
    }
};

// Parent levels over `nchild` children whose boxes sit in shared memory
// (src), for at most max_levels levels or up to the root; ping-pongs src and
// dst and leaves the last level's boxes in src.
__device__ __forceinline__ void smem_levels(const RadvArgs& A, uint8_t* boxes, float*& mn_src, float*& mx_src,
                                            float*& mn_dst, float*& mx_dst, uint32_t& nchild, uint32_t& child_base,
                                            uint32_t& lvl, uint32_t max_levels) {
    for (uint32_t j = 1; j <= max_levels && lvl > 0; ++j) {
        const uint32_t plvl = lvl - 1;
        const uint32_t np = (nchild + 3) / 4;
        const uint32_t pbase = child_base >> 2;
        for (uint32_t t = threadIdx.x; t < np; t += kT) {
            float umn[3], umx[3];
            make_parent(boxes, A.offs[plvl] + pbase + t, A.offs[lvl] + child_base + 4 * t, min(4u, nchild - 4 * t),
                        SmemChildren{mn_src + 12 * t, mx_src + 12 * t}, umn, umx);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn_dst[3 * t + k] = umn[k];
                mx_dst[3 * t + k] = umx[k];
            }
        }
        __syncthreads();
        float* tn = mn_src;
        mn_src = mn_dst;
        mn_dst = tn;
        float* tx = mx_src;
        mx_src = mx_dst;
        mx_dst = tx;
        nchild = np;
        child_base = pbase;
        lvl = plvl;
    }
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

// STAGE: the warp-staged leaf round (coalesced); without it each lane reads
// its own triangle and writes its own node parts, which has fewer dependent
// steps and is faster for a one-block image.
template <int LB, bool STAGE>
__global__ void __launch_bounds__(kT, LB == 256 ? 6 : 4) k_radv(RadvArgs A) {
    static_assert(LB == 64 || LB == 256 || LB == 1024, "a block's subtree is a complete 4-ary tree");
    constexpr uint32_t kInLevels = LB == 1024 ? 5u : LB == 256 ? 4u : 3u;  // log4(LB)
    // leaf-level boxes (LB) and the first parent level (LB/4) ping-pong
    __shared__ float s_mn0[LB * 3], s_mx0[LB * 3];
    __shared__ float s_mn1[LB / 4 * 3], s_mx1[LB / 4 * 3];
    // per warp: its 32 triangles' vertices as read, and their bounds
    // (rows padded: a lane may read 3 floats past its warp's last triangle;
    // box rows at a stride of 7 floats, which keeps the lanes on distinct banks)
    __shared__ float s_raw[STAGE ? kT / 32 : 1][32 * 9 + 4];
    __shared__ float s_tbox[STAGE ? kT / 32 : 1][32 * 7];
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
    // A round is kT consecutive triangles, 32 per warp.  Each warp reads its
    // triangles' 1,152 B with coalesced loads into shared memory, then
    // writes their 64-B triangle nodes (2 KB) and the 8 leaf box nodes over
    // them (1 KB) as runs of 16 B per lane, consecutive lanes on consecutive
    // addresses.
    const uint32_t w = threadIdx.x >> 5;
    float* raw = s_raw[STAGE ? w : 0];
    float* tbox = s_tbox[STAGE ? w : 0];
    const uint32_t lb0 = blockIdx.x * LB;
    const uint32_t nlb = min(uint32_t(LB), leaf_cnt - lb0);
    const uint32_t tend = min(A.n, (lb0 + nlb) * 4u);  // end of this block's triangles
    // rounds that hold any of this block's triangles (at most 4*LB/kT; the
    // same for every thread)
    const uint32_t rounds = (nlb * 4u + kT - 1) / kT;
    // staged rounds read the next round's triangles into registers while the
    // current round is written out
    float pf[9];
    if constexpr (STAGE) {
        const uint32_t tb0 = lb0 * 4u + w * 32;
        if (tb0 < tend) {
            const uint32_t nt0 = min(32u, tend - tb0);
            const float* src = A.tri9 + 9ull * tb0;
#pragma unroll
            for (uint32_t j = 0; j < 9; ++j) {
                const uint32_t q = j * 32 + lane;
                pf[j] = q < 9 * nt0 ? __ldg(src + q) : 0.0f;
            }
        }
    }
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t wl = r * kT + w * 32;  // first triangle of this warp, within the block
        const uint32_t tb = lb0 * 4u + wl;    // the same, in the mesh
        if (tb >= tend) continue;             // the warp holds no triangle and no leaf box
        const uint32_t nt = min(32u, tend - tb);
        if constexpr (!STAGE) {
            float tmn[3] = {qn, qn, qn}, tmx[3] = {qn, qn, qn};
            const uint32_t ti = tb + lane;
            const bool valid = lane < nt;
            if (valid) {
                const float* v = A.tri9 + 9ull * ti;
                float f[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) f[q] = __ldg(v + q);
                uint4* o = reinterpret_cast<uint4*>(trin + 64ull * ti);
                o[0] = make_uint4(__float_as_uint(f[0]), __float_as_uint(f[1]), __float_as_uint(f[2]),
                                  __float_as_uint(f[3]));
                o[1] = make_uint4(__float_as_uint(f[4]), __float_as_uint(f[5]), __float_as_uint(f[6]),
                                  __float_as_uint(f[7]));
                o[2] = make_uint4(__float_as_uint(f[8]), 0u, 0u, 0u);
                o[3] = make_uint4(ti, RQ_RADV_GEOMETRY_OPAQUE, 0u, RQ_RADV_BARYCENTRICS_CONTROL_DEFAULT);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    tmn[k] = fminf(f[k], fminf(f[3 + k], f[6 + k]));
                    tmx[k] = fmaxf(f[k], fmaxf(f[3 + k], f[6 + k]));
                }
            }
            // this lane's quarter of its leaf box node: child id, child box
            // and one dword of the zero tail
            const uint32_t lbl = (wl + lane) >> 2;
            const uint32_t c = lane & 3u;
            if (lbl < nlb) {
                uint8_t* nd = boxes + 128ull * (A.offs[leaf_lvl] + lb0 + lbl);
                reinterpret_cast<uint32_t*>(nd)[c] =
                    valid ? ((A.total_boxes * 128u + ti * 64u) >> 3) | RQ_RADV_NODE_TRIANGLE : RQ_RADV_INVALID_NODE;
                float2* b = reinterpret_cast<float2*>(nd + 16 + 24 * c);
                b[0] = make_float2(tmn[0], tmn[1]);
                b[1] = make_float2(tmn[2], tmx[0]);
                b[2] = make_float2(tmx[1], tmx[2]);
                reinterpret_cast<uint32_t*>(nd + 112)[c] = 0u;
            }
            // the leaf box's bounds, children in order 0..3
            const uint32_t g0 = lane & ~3u;
            float umn[3] = {1e30f, 1e30f, 1e30f}, umx[3] = {-1e30f, -1e30f, -1e30f};
#pragma unroll
            for (int cc = 0; cc < 4; ++cc)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    umn[k] = fminf(umn[k], __shfl_sync(0xffffffffu, tmn[k], g0 + cc));
                    umx[k] = fmaxf(umx[k], __shfl_sync(0xffffffffu, tmx[k], g0 + cc));
                }
            if (c == 0u && lbl < nlb) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    s_mn0[3 * lbl + k] = umn[k];
                    s_mx0[3 * lbl + k] = umx[k];
                }
            }
        } else {
#pragma unroll
            for (uint32_t j = 0; j < 9; ++j) {
                const uint32_t q = j * 32 + lane;
                if (q < 9 * nt) raw[q] = pf[j];
            }
            __syncwarp();
            if (r + 1 < rounds && tb + kT < tend) {
                const uint32_t ntn = min(32u, tend - (tb + kT));
                const float* src = A.tri9 + 9ull * (tb + kT);
#pragma unroll
                for (uint32_t j = 0; j < 9; ++j) {
                    const uint32_t q = j * 32 + lane;
                    pf[j] = q < 9 * ntn ? __ldg(src + q) : 0.0f;
                }
            }
            // this lane's triangle bounds (qNaN for a slot past the mesh's end)
            float tmn[3] = {qn, qn, qn}, tmx[3] = {qn, qn, qn};
            if (lane < nt) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float a = raw[9 * lane + k], b = raw[9 * lane + 3 + k], c = raw[9 * lane + 6 + k];
                    tmn[k] = fminf(a, fminf(b, c));
                    tmx[k] = fmaxf(a, fmaxf(b, c));
                }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                tbox[7 * lane + k] = tmn[k];
                tbox[7 * lane + 3 + k] = tmx[k];
            }
            __syncwarp();
            // triangle nodes: 16-B part p of triangle t, four triangles per 4 lanes
            {
                // every lane reads four floats (from vertex float 0, 4 or 8)
                // and keeps what its part needs, so the lanes do not diverge
                const uint32_t p = lane & 3u;
                const uint32_t pk = p < 2u ? 4u * p : 8u;
#pragma unroll
                for (uint32_t q = 0; q < 4; ++q) {
                    const uint32_t t = 8 * q + (lane >> 2);
                    if (t < nt) {
                        const float* f = raw + 9 * t + pk;
                        const uint32_t a0 = __float_as_uint(f[0]), a1 = __float_as_uint(f[1]),
                                       a2 = __float_as_uint(f[2]), a3 = __float_as_uint(f[3]);
                        const uint4 v =
                            p < 2u ? make_uint4(a0, a1, a2, a3)
                                   : p == 2u ? make_uint4(a0, 0u, 0u, 0u)
                                             : make_uint4(tb + t, RQ_RADV_GEOMETRY_OPAQUE, 0u,
                                                          RQ_RADV_BARYCENTRICS_CONTROL_DEFAULT);
                        reinterpret_cast<uint4*>(trin + 64ull * (tb + t))[p] = v;
                    }
                }
            }
            // leaf box nodes: 16-B part F of node d (ids, six runs of the four
            // child boxes, zero tail), eight lanes per node
            {
                const uint32_t F = lane & 7u;
#pragma unroll
                for (uint32_t q = 0; q < 2; ++q) {
                    const uint32_t d = 4 * q + (lane >> 3);
                    const uint32_t lbl = wl / 4 + d;  // leaf box within block
                    if (lbl < nlb) {
                        uint4 v;
                        if (F == 0u) {
                            uint32_t id[4];
#pragma unroll
                            for (uint32_t c = 0; c < 4; ++c) {
                                const uint32_t t = 4 * d + c;
                                id[c] = t < nt ? ((A.total_boxes * 128u + (tb + t) * 64u) >> 3) | RQ_RADV_NODE_TRIANGLE
                                               : RQ_RADV_INVALID_NODE;
                            }
                            v = make_uint4(id[0], id[1], id[2], id[3]);
                        } else if (F == 7u) {
                            v = make_uint4(0u, 0u, 0u, 0u);
                        } else {
                            // floats e..e+3 of the four child boxes (6 floats each)
                            uint32_t x[4];
#pragma unroll
                            for (uint32_t i = 0; i < 4; ++i) {
                                const uint32_t e = 4 * (F - 1) + i;
                                x[i] = __float_as_uint(tbox[7 * (4 * d + e / 6) + e % 6]);
                            }
                            v = make_uint4(x[0], x[1], x[2], x[3]);
                        }
                        reinterpret_cast<uint4*>(boxes + 128ull * (A.offs[leaf_lvl] + lb0 + lbl))[F] = v;
                    }
                }
            }
            // leaf box bounds for the parent levels: children in order 0..3 (a
            // missing child's qNaN is skipped by fminf/fmaxf)
            if (lane < 8u && wl / 4 + lane < nlb) {
                float umn[3] = {1e30f, 1e30f, 1e30f}, umx[3] = {-1e30f, -1e30f, -1e30f};
#pragma unroll
                for (int c = 0; c < 4; ++c)
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        umn[k] = fminf(umn[k], tbox[7 * (4 * lane + c) + k]);
                        umx[k] = fmaxf(umx[k], tbox[7 * (4 * lane + c) + 3 + k]);
                    }
                const uint32_t lbl = wl / 4 + lane;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    s_mn0[3 * lbl + k] = umn[k];
                    s_mx0[3 * lbl + k] = umx[k];
                }
            }
            __syncwarp();  // the next round rewrites raw and tbox
        }
    }
    __syncthreads();

    // ---- in-block levels (log4(LB))
    uint32_t nchild = nlb;      // children at the current level in this block
    uint32_t child_base = lb0;  // first child index within its level
    uint32_t lvl = leaf_lvl;    // level of the children
    smem_levels(A, boxes, cmn_src, cmx_src, cmn_dst, cmx_dst, nchild, child_base, lvl, kInLevels);

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
    // every other block has taken its ticket: ready it for the next launch
    if (threadIdx.x == 0) *A.ticket = 0u;
    __threadfence();
    // level `lvl` holds gridDim.x nodes whose boxes are in A.top[2b], A.top[2b+1];
    // parents through global memory while there are more than LB of them,
    // then the rest of the way in shared memory
    float4* src = A.top;
    float4* dst = A.top + 2 * gridDim.x;
    nchild = A.counts[lvl];
    while (nchild > uint32_t(LB)) {
        const uint32_t plvl = lvl - 1;
        const uint32_t np = A.counts[plvl];
        for (uint32_t t = threadIdx.x; t < np; t += kT) {
            float umn[3], umx[3];
            make_parent(boxes, A.offs[plvl] + t, A.offs[lvl] + 4 * t, min(4u, nchild - 4 * t),
                        GlobalChildren{src + 8 * t}, umn, umx);
            __stcg(dst + 2 * t, make_float4(umn[0], umn[1], umn[2], 0.0f));
            __stcg(dst + 2 * t + 1, make_float4(umx[0], umx[1], umx[2], 0.0f));
        }
        __syncthreads();  // the block's own global writes are visible to it after the barrier
        float4* tmp = src;
        src = dst;
        dst = tmp;
        nchild = np;
        lvl = plvl;
    }
    for (uint32_t t = threadIdx.x; t < nchild; t += kT) {
        const float4 a = __ldcg(src + 2 * t), b = __ldcg(src + 2 * t + 1);
        s_mn0[3 * t] = a.x;
        s_mn0[3 * t + 1] = a.y;
        s_mn0[3 * t + 2] = a.z;
        s_mx0[3 * t] = b.x;
        s_mx0[3 * t + 1] = b.y;
        s_mx0[3 * t + 2] = b.z;
    }
    __syncthreads();
    cmn_src = s_mn0;
    cmx_src = s_mx0;
    cmn_dst = s_mn1;
    cmx_dst = s_mx1;
    child_base = 0;
    smem_levels(A, boxes, cmn_src, cmx_src, cmn_dst, cmx_dst, nchild, child_base, lvl, 32u);
    if (threadIdx.x == 0) {
        float mn[3] = {cmn_src[0], cmn_src[1], cmn_src[2]};
        float mx[3] = {cmx_src[0], cmx_src[1], cmx_src[2]};
        write_header(A, mn, mx);
    }
}

// Launches the build; returns this launch's own error (cudaLaunchKernel
// reports the launch it was given, not an earlier call's pending error).
cudaError_t launch_radv(const RadvArgs& a, uint32_t leaf_cnt, cudaStream_t st) {
    const uint32_t lb = radv_leaf_boxes(leaf_cnt);
    const uint32_t blocks = radv_blocks(leaf_cnt, lb);
    const void* k = lb == 1024u  ? reinterpret_cast<const void*>(k_radv<1024, true>)
                    : lb == 256u ? reinterpret_cast<const void*>(k_radv<256, true>)
                    : blocks > 1 ? reinterpret_cast<const void*>(k_radv<64, true>)
                                 : reinterpret_cast<const void*>(k_radv<64, false>);
    RadvArgs arg = a;
    void* args[] = {&arg};
    return cudaLaunchKernel(k, dim3(blocks), dim3(kT), args, 0, st);
}

}  // namespace

// ---------------------------------------------------------------------------
// Allocation-free RADV build.  Some callers own every byte of device memory
// they use — they size their buffers up front from their own pool or budget
// and cannot let a library call cudaMalloc / cudaFree, which synchronise the
// whole device and can fail mid-frame.  This variant takes only the vertex
// buffer and the image buffer from the caller; its scratch (the finishing
// ticket and two boxes per block, twice, for the top levels) lives in the static
// device array below, sized for at most RQ_RADV_NOALLOC_MAX_TRIANGLES
// triangles (256 KiB).  Every GPU that loads librq.so holds the array until
// the process exits.  The array starts at zero and every build leaves the
// ticket at zero.  Host code cannot pass the array's name to a kernel (on
// the host it names a stand-in, not device memory), so every call looks up
// the array's device address on the current device with
// cudaGetSymbolAddress, which allocates nothing.  Looking it up each time
// (rather than caching it per device) stays right after a device reset,
// which gives the array a new address.
// The most blocks a build of at most RQ_RADV_NOALLOC_MAX_TRIANGLES takes:
// 1024-leaf-box subtrees at the largest size, fewer than 4 * kLargeBlocksMin
// of 256 leaf boxes, or at most kSmallBlocksMax of 64.
constexpr uint32_t kNoallocBlocks = std::max<uint32_t>(
    {(RQ_RADV_NOALLOC_MAX_TRIANGLES / 4 + 1023u) / 1024u, 4 * kLargeBlocksMin, kSmallBlocksMax});
static __device__ __align__(256) unsigned char rq_radv_noalloc_scratch[256 + 4 * sizeof(float4) * kNoallocBlocks];

extern "C" int rq_build_radv_noalloc(const float* tri9, uint32_t num_triangles, void* as_image, uint64_t as_bytes,
                                     rq_stream stream) {
    if (!tri9 || !as_image || num_triangles == 0) return RQ_ERR_INVALID_ARG;
    if (num_triangles > RQ_RADV_NOALLOC_MAX_TRIANGLES) return RQ_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(as_image) & 15u) || (reinterpret_cast<uintptr_t>(tri9) & 3u))
        return RQ_ERR_INVALID_ARG;
    rq_radv_layout L;
    if (rq_radv_layout_get(num_triangles, &L) != RQ_OK) return RQ_ERR_UNSUPPORTED;
    if (as_bytes < L.total_as_size) return RQ_ERR_SIZE;
    // the array's device address on the current device (the first call on a
    // device, or after a reset, also loads the library's device code there)
    void* base = nullptr;
    const cudaError_t ge = cudaGetSymbolAddress(&base, rq_radv_noalloc_scratch);
    if (ge != cudaSuccess || !base) {
        if (ge == cudaErrorNoDevice || ge == cudaErrorInsufficientDriver) return RQ_ERR_NO_DEVICE;
        return RQ_ERR_CUDA;
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
    const uint32_t leaf_cnt = L.level_counts[L.num_levels - 1];
    return launch_radv(a, leaf_cnt, st) == cudaSuccess ? RQ_OK : RQ_ERR_CUDA;
}

int rq_launch_radv(rq_ctx* ctx, const float* tri9, uint32_t n, void* img, const rq_radv_layout& L, cudaStream_t st,
                   bool refit) {
    const uint32_t leaf_cnt = L.level_counts[L.num_levels - 1];
    const uint32_t blocks = radv_blocks(leaf_cnt, radv_leaf_boxes(leaf_cnt));
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
    a.ticket = ctx->d_err + RQ_CTX_RADV_TICKET;
    a.top = reinterpret_cast<float4*>(static_cast<char*>(ctx->scratch) + 256);
    a.size = L.total_as_size;
    a.check_header = refit ? 1u : 0u;
    a.err = ctx->d_err;
    return rq_cuda_status(ctx, launch_radv(a, leaf_cnt, st), "radv build launch");
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
