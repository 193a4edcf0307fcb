// k_sort.cu — stable LSD radix sort of (key, value) pairs in the onesweep
// form (Adinets & Merrill 2022): one upfront histogram pass for every digit
// position, then one kernel per 8-bit digit that ranks a 4608-key tile,
// resolves the tile's global digit offsets by decoupled look-back over the
// preceding tiles, and scatters through shared memory.  Also a single-pass
// decoupled look-back exclusive scan over uint32.
//
// Tiles are claimed in launch order through an atomic ticket, so a tile only
// ever waits on tiles whose blocks are already running; every wait is
// bounded (RQ_SPIN_LIMIT) and records RQ_DERR_* on the context's error word.
#include "rq_device.cuh"
#include "rq_internal.h"

namespace {

constexpr int kThreads = 256;
// 18 keys per thread: the 2.5M-key sort of a 2,499,848-triangle build is 543
// tiles, within one wave of 4 blocks on 148 SMs (16 keys: 611 tiles, a second
// wave of 19; the build 1.031 -> 1.016 ms)
constexpr int kItems = 18;
constexpr int kTile = kThreads * kItems;  // 4608 keys
constexpr int kRadix = 256;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
constexpr uint32_t kSpinLimit = 1u << 21;

__global__ void __launch_bounds__(kThreads) k_hist(const uint32_t* __restrict__ keys, uint32_t n,
                                                   uint32_t passes, uint32_t* __restrict__ hist) {
    // one private histogram per warp pair to thin out shared-atomic collisions
    __shared__ uint32_t sh[4][4][kRadix];
    uint32_t* flat = &sh[0][0][0];
    for (int i = threadIdx.x; i < 4 * 4 * kRadix; i += kThreads) flat[i] = 0;
    __syncthreads();
    const int copy = (threadIdx.x >> 6) & 3;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        uint32_t k = keys[i];
        for (uint32_t p = 0; p < passes; ++p) atomicAdd(&sh[copy][p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kRadix; i += kThreads) {
        int p = i >> 8, d = i & 255;
        uint32_t v = sh[0][p][d] + sh[1][p][d] + sh[2][p][d] + sh[3][p][d];
        if (v) atomicAdd(&hist[i], v);
    }
}

// Block-wide exclusive scan of one value per thread (256 threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* s_warp, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kWarps ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kWarps) s_warp[lane] = w;  // inclusive warp prefix
    }
    __syncthreads();
    uint32_t warp_prefix = warp ? s_warp[warp - 1] : 0u;
    if (total) *total = s_warp[kWarps - 1];
    uint32_t r = warp_prefix + x - v;
    __syncthreads();
    return r;
}

// Exclusive scan of each pass's 256 bins, in place.
__global__ void __launch_bounds__(kThreads) k_hist_scan(uint32_t* hist) {
    __shared__ uint32_t s_warp[kWarps];
    uint32_t* h = hist + blockIdx.x * kRadix;
    uint32_t v = h[threadIdx.x];
    uint32_t ex = block_exclusive_scan(v, s_warp, nullptr);
    h[threadIdx.x] = ex;
}

// 4 blocks per SM (64 registers): the 2.5M-triangle build 1.047 -> 1.038 ms
// against 3 blocks at 80 registers; 5 blocks spill more and are slower
__global__ void __launch_bounds__(kThreads, 4) k_onesweep(const uint32_t* __restrict__ keys_in,
                                                       const uint32_t* __restrict__ vals_in,
                                                       uint32_t* __restrict__ keys_out,
                                                       uint32_t* __restrict__ vals_out, uint32_t n,
                                                       uint32_t shift, const uint32_t* __restrict__ pass_base,
                                                       uint32_t* status, uint32_t* tile_ctr, uint32_t* err) {
    __shared__ uint32_t s_cnt[kWarps][kRadix];
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_dig_off[kRadix];
    __shared__ uint32_t s_glob[kRadix];
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint32_t s_tile;

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kThreads) (&s_cnt[0][0])[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t tile_base = tile * kTile;

    uint32_t key[kItems], val[kItems], rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint32_t idx = tile_base + warp * (32 * kItems) + j * 32 + lane;
        bool valid = idx < n;
        key[j] = valid ? keys_in[idx] : 0u;
        val[j] = valid ? vals_in[idx] : 0u;
    }
    // Rank within the warp, item by item in tile order: peers with the same
    // digit get consecutive ranks in lane order (stable).
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint32_t idx = tile_base + warp * (32 * kItems) + j * 32 + lane;
        bool valid = idx < n;
        uint32_t act = __ballot_sync(0xffffffffu, valid);
        rank[j] = 0;
        if (valid) {
            uint32_t d = (key[j] >> shift) & 255u;
            uint32_t peers = __match_any_sync(act, d);
            int leader = __ffs(peers) - 1;
            uint32_t below = __popc(peers & ((1u << lane) - 1u));
            uint32_t base = 0;
            if (lane == leader) {
                base = s_cnt[warp][d];
                s_cnt[warp][d] = base + __popc(peers);
            }
            base = __shfl_sync(peers, base, leader);
            rank[j] = base + below;
        }
        __syncwarp();
    }
    __syncthreads();
    // Per digit (thread = digit): warp-exclusive offsets and tile total.
    const uint32_t d = threadIdx.x;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        uint32_t c = s_cnt[w][d];
        s_cnt[w][d] = run;
        run += c;
    }
    const uint32_t total = run;
    // publish the tile aggregate early so successors can proceed
    uint32_t* my_status = status + size_t(tile) * kRadix;
    if (tile != 0) rq::st_release(&my_status[d], kFlagAgg | total);
    uint32_t dig_off = block_exclusive_scan(total, s_warp, nullptr);
    s_dig_off[d] = dig_off;
    // decoupled look-back for this digit
    uint32_t glob;
    if (tile == 0) {
        glob = pass_base[d];
        rq::st_release(&my_status[d], kFlagPrefix | (glob + total));
    } else {
        // windowed: the statuses of the kWindow nearest unvisited
        // predecessors are read at once (relaxed loads: each count shares
        // its word with its flag, and nothing else the predecessor wrote is
        // read), then walked nearest first until an inclusive prefix; a
        // predecessor not yet published ends the window and is read again.
        // Measured against one tile per read: the 2.5M-triangle build went
        // from 1.051 to 1.042 ms.
        constexpr int kWindow = 8;
        uint32_t acc = 0, spins = 0;
        int t = int(tile) - 1;
        for (;;) {
            uint32_t st[kWindow];
#pragma unroll
            for (int q = 0; q < kWindow; ++q)
                st[q] = t - q >= 0 ? rq::ld_relaxed(&status[size_t(t - q) * kRadix + d]) : 0u;
            int used = 0;
            bool done = false;
#pragma unroll
            for (int q = 0; q < kWindow; ++q) {
                if (done || used < q) continue;  // stopped earlier in this window
                const uint32_t flag = st[q] & ~kValueMask;
                if (flag == 0u) continue;        // not yet published: read again from here
                acc += st[q] & kValueMask;
                used = q + 1;
                done = flag == kFlagPrefix;
            }
            if (done) break;
            if (used == 0 && ++spins > kSpinLimit) {
                rq::set_err(err, RQ_DERR_SORT_LOOKBACK);
                break;
            }
            t -= used;
        }
        glob = acc;
        rq::st_release(&my_status[d], kFlagPrefix | (acc + total));
    }
    s_glob[d] = glob;
    __syncthreads();
    // scatter into shared memory in digit order
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
        uint32_t idx = tile_base + warp * (32 * kItems) + j * 32 + lane;
        if (idx < n) {
            uint32_t dj = (key[j] >> shift) & 255u;
            uint32_t pos = s_dig_off[dj] + s_cnt[warp][dj] + rank[j];
            s_keys[pos] = key[j];
            s_vals[pos] = val[j];
        }
    }
    __syncthreads();
    const uint32_t tile_n = n - tile_base < uint32_t(kTile) ? n - tile_base : uint32_t(kTile);
    for (uint32_t i = threadIdx.x; i < tile_n; i += kThreads) {
        uint32_t k = s_keys[i];
        uint32_t dk = (k >> shift) & 255u;
        uint32_t g = s_glob[dk] + (i - s_dig_off[dk]);
        keys_out[g] = k;
        vals_out[g] = s_vals[i];
    }
}

// ------------------------------------------------------------------ scan
constexpr int kScanItems = 8;
constexpr int kScanTile = kThreads * kScanItems;

// GATHER: the i-th input is in[order[i]].
template <bool GATHER>
__global__ void __launch_bounds__(kThreads) k_scan(const uint32_t* __restrict__ in, const uint32_t* __restrict__ order,
                                                   uint32_t* __restrict__ out, uint32_t n, uint32_t* status,
                                                   uint32_t* tile_ctr, uint32_t* err) {
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint32_t s_tile, s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? in[GATHER ? order[base + i] : base + i] : 0u;
        sum += v[i];
    }
    uint32_t total;
    uint32_t ex = block_exclusive_scan(sum, s_warp, &total);
    if (threadIdx.x < 32) {
        // warp-wide decoupled look-back: 32 predecessors per step; the
        // nearest one with its inclusive prefix ends the walk
        const uint32_t lane = threadIdx.x;
        if (tile == 0) {
            if (lane == 0) {
                rq::st_release(&status[0], kFlagPrefix | total);
                s_prefix = 0;
            }
        } else {
            if (lane == 0) rq::st_release(&status[tile], kFlagAgg | total);
            uint32_t acc = 0, spins = 0;
            for (int t0 = int(tile) - 1;; t0 -= 32) {
                const int t = t0 - int(lane);
                uint32_t st = kFlagPrefix;  // before tile 0: an inclusive prefix of 0
                if (t >= 0) {
                    for (;;) {
                        st = rq::ld_acquire(&status[t]);
                        if (st & ~kValueMask) break;
                        if (++spins > kSpinLimit) {
                            rq::set_err(err, RQ_DERR_SCAN_LOOKBACK);
                            st = kFlagPrefix;
                            break;
                        }
                    }
                }
                const uint32_t pm = __ballot_sync(0xffffffffu, (st & ~kValueMask) == kFlagPrefix);
                uint32_t val = st & kValueMask;
                if (pm && int(lane) > __ffs(pm) - 1) val = 0u;
                acc += __reduce_add_sync(0xffffffffu, val);
                if (pm) break;
            }
            if (lane == 0) {
                rq::st_release(&status[tile], kFlagPrefix | (acc + total));
                s_prefix = acc;
            }
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + ex;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

}  // namespace

uint32_t rq_sort_tiles(uint32_t n) { return (n + kTile - 1) / kTile; }
uint32_t rq_scan_tiles(uint32_t n) { return (n + kScanTile - 1) / kScanTile; }

int rq_launch_sort(rq_ctx* ctx, BuildScratch& s, uint32_t n, uint32_t bits, cudaStream_t st, int* result_buf) {
    const uint32_t passes = (bits + 7) / 8;
    const uint32_t tiles = rq_sort_tiles(n);
    cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * 4 * kRadix, st);
    cudaMemsetAsync(s.sort_status, 0, sizeof(uint32_t) * size_t(passes) * tiles * kRadix, st);
    uint32_t hist_blocks = tiles < uint32_t(2 * ctx->num_sms) ? tiles : uint32_t(2 * ctx->num_sms);
    k_hist<<<hist_blocks, kThreads, 0, st>>>(s.keys[0], n, passes, s.hist);
    k_hist_scan<<<passes, kThreads, 0, st>>>(s.hist);
    for (uint32_t p = 0; p < passes; ++p) {
        int a = int(p & 1), b = 1 - a;
        k_onesweep<<<tiles, kThreads, 0, st>>>(s.keys[a], s.vals[a], s.keys[b], s.vals[b], n, 8 * p,
                                               s.hist + kRadix * p, s.sort_status + size_t(p) * tiles * kRadix,
                                               s.tile_ctr + p, ctx->d_err);
    }
    *result_buf = int(passes & 1);
    return rq_cuda_status(ctx, cudaGetLastError(), "radix sort launch");
}

void rq_launch_scan(rq_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* status,
                    uint32_t* tile_ctr, cudaStream_t st, const uint32_t* order) {
    const uint32_t tiles = rq_scan_tiles(n);
    cudaMemsetAsync(status, 0, sizeof(uint32_t) * tiles, st);
    if (order)
        k_scan<true><<<tiles, kThreads, 0, st>>>(in, order, out, n, status, tile_ctr, ctx->d_err);
    else
        k_scan<false><<<tiles, kThreads, 0, st>>>(in, nullptr, out, n, status, tile_ctr, ctx->d_err);
}
