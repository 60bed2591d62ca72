// Onesweep LSD radix sort pieces shared by the LBVH build (Morton keys) and the
// renderer (ray-queue coherence keys): the per-pass digit-offset scan and the
// digit pass itself (tile ranking with warp match/popc scans, decoupled look-back
// with a bounded wait, staged scatter). The element count may live on the device
// (n_ptr): tiles that start past it leave at once (no later tile needs them).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "cpt.h"

namespace cpt {

constexpr int kRadix = 256;
constexpr int kSortBlock = 256;  // one thread per digit in the per-tile digit work
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096 keys per tile
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kValueMask = (1u << 30) - 1;
constexpr uint32_t kLookbackPolls = 1u << 22;  // default poll limit of one tile's look-back

// Look-back wait settings of one digit pass: the poll limit, and (a test of the
// failure path only) whether the pass's tile 0 withholds its published counts, so
// that every look-back reaching it waits out the limit and reports a timeout.
struct SortWait {
    uint32_t poll_limit = kLookbackPolls;
    uint32_t withhold_tile0 = 0;
};

// Exclusive prefix of each pass's 256 digit counts (one block per pass).
static __global__ void __launch_bounds__(kRadix) k_scan_offsets(const uint32_t* __restrict__ hist,
                                                         uint32_t* __restrict__ offsets)
{
    __shared__ uint32_t s_warp[kRadix / 32];
    const uint32_t* h = hist + blockIdx.x * kRadix;
    uint32_t v = h[threadIdx.x];
    uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kRadix / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < kRadix / 32) s_warp[lane] = w;
    }
    __syncthreads();
    uint32_t before = warp ? s_warp[warp - 1] : 0;
    offsets[blockIdx.x * kRadix + threadIdx.x] = before + x - v;
}

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) { return *reinterpret_cast<const volatile uint32_t*>(p); }
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) { *reinterpret_cast<volatile uint32_t*>(p) = v; }

template <typename K>
constexpr size_t onesweep_smem() { return (size_t)kSortTile * sizeof(K) + (size_t)kSortTile * 4 + (size_t)kSortWarps * kRadix * 4 + 2 * kRadix * 4; }

// One digit pass. Tiles are claimed in launch order through tile_counter, so a
// tile only ever waits on tiles already owned by running blocks (which publish
// their own counts before they wait): the look-back always completes; the poll
// bound (wait.poll_limit polls of one tile, then CPT_STATUS_TIMEOUT and the tile
// goes on with the prefix it has) is a guard, not a scheduling assumption. Output
// positions stay inside [0, n) whatever prefix a timed-out tile uses, because a
// prefix read from the look-back never exceeds the true one.
template <typename K, bool kFirst>
#ifndef CPT_SORT_MIN_BLOCKS
#define CPT_SORT_MIN_BLOCKS 3  // 80 registers: three 4096-key tiles per SM (0.63 vs 0.67 ms per 5.2 M-key sort)
#endif
__global__ void __launch_bounds__(kSortBlock, CPT_SORT_MIN_BLOCKS) k_onesweep(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                         K* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n_arg,
                                                         const uint32_t* __restrict__ n_ptr,
                                                         int shift, const uint32_t* __restrict__ offsets,
                                                         uint32_t* __restrict__ lookback,
                                                         uint32_t* __restrict__ tile_counter,
                                                         uint32_t* __restrict__ status, SortWait wait = SortWait())
{
    extern __shared__ __align__(16) unsigned char smem[];
    K* s_keys = reinterpret_cast<K*>(smem);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_keys + kSortTile);
    uint32_t* s_hist = s_vals + kSortTile;       // [warp][digit]
    uint32_t* s_off = s_hist + kSortWarps * kRadix;  // tile-local exclusive offset per digit
    uint32_t* s_base = s_off + kRadix;           // global output base per digit
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_wsum[kSortWarps];

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_counter, 1u);
    for (uint32_t i = tid; i < kSortWarps * kRadix; i += kSortBlock) s_hist[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t tile_start = tile * kSortTile;
    const uint32_t n = n_ptr ? *n_ptr : n_arg;
    if (tile_start >= n && tile > 0) return;  // empty tile: every later tile is empty too
    const uint32_t wbase = tile_start + warp * (kSortItems * 32);

    K key[kSortItems];
    uint32_t val[kSortItems];
    uint32_t rank[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = wbase + k * 32 + lane;
        bool valid = idx < n;
        key[k] = valid ? kin[idx] : (K)0;
        val[k] = kFirst ? idx : (valid ? vin[idx] : 0u);
    }
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t* my_hist = s_hist + warp * kRadix;
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = wbase + k * 32 + lane;
        uint32_t dig = idx < n ? (uint32_t)((key[k] >> shift) & 0xFF) : kRadix;
        unsigned peers = __match_any_sync(0xFFFFFFFFu, dig);
        uint32_t cnt = dig < kRadix ? my_hist[dig] : 0u;
        rank[k] = cnt + __popc(peers & lt_mask);
        __syncwarp();
        if (dig < kRadix && lane == (uint32_t)(__ffs(peers) - 1)) my_hist[dig] = cnt + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Per digit (thread tid = digit): exclusive prefix over warps, tile count.
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        uint32_t c = s_hist[w * kRadix + tid];
        s_hist[w * kRadix + tid] = count;
        count += c;
    }
    // Publish this tile's count as early as possible.
    if (tile != 0 || !wait.withhold_tile0)
        st_volatile(&lookback[(size_t)tile * kRadix + tid], (tile == 0 ? kFlagInc : kFlagAgg) | count);

    // Tile-local exclusive scan of the digit counts (warp shuffles + warp totals).
    uint32_t x = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    uint32_t before = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) before += (w < (int)warp) ? s_wsum[w] : 0u;
    s_off[tid] = before + x - count;

    // Decoupled look-back over the preceding tiles for this digit.
    uint32_t prefix = 0;
    if (tile > 0) {
        int j = (int)tile - 1;
        uint32_t polls = 0;
        bool timed_out = false;
        while (j >= 0) {
            uint32_t v = ld_volatile(&lookback[(size_t)j * kRadix + tid]);
            uint32_t f = v & ~kValueMask;
            if (f == 0) {
                if (++polls > wait.poll_limit) { timed_out = true; break; }
                if (polls > 32) __nanosleep(100);
                continue;
            }
            prefix += v & kValueMask;
            if (f == kFlagInc) break;
            --j;
        }
        if (timed_out) atomicOr(status, CPT_STATUS_TIMEOUT);
        st_volatile(&lookback[(size_t)tile * kRadix + tid], kFlagInc | ((prefix + count) & kValueMask));
    }
    s_base[tid] = offsets[tid] + prefix;
    __syncthreads();

    // Stage the tile in local sorted order, then write runs of equal digits.
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t idx = wbase + k * 32 + lane;
        if (idx < n) {
            uint32_t dig = (uint32_t)((key[k] >> shift) & 0xFF);
            uint32_t pos = s_off[dig] + my_hist[dig] + rank[k];
            s_keys[pos] = key[k];
            s_vals[pos] = val[k];
        }
    }
    __syncthreads();
    const uint32_t tile_n = min((uint32_t)kSortTile, n - tile_start);
    for (uint32_t i = tid; i < tile_n; i += kSortBlock) {
        K kk = s_keys[i];
        uint32_t dig = (uint32_t)((kk >> shift) & 0xFF);
        uint32_t o = s_base[dig] + (i - s_off[dig]);
        kout[o] = kk;
        vout[o] = s_vals[i];
    }
}


}  // namespace cpt
