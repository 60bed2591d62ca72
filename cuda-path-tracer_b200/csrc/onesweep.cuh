// Onesweep LSD radix sort pieces shared by the LBVH build (Morton keys) and the
// renderer (ray-queue coherence keys): the per-pass digit-offset scan and the
// digit pass itself (tile ranking with warp match/popc scans, decoupled look-back
// with a bounded wait, staged scatter). The element count may live on the device
// (n_ptr): tiles that start past it leave at once (no later tile needs them).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "cpt.h"
#include "cpt_internal.h"

namespace cpt {

constexpr int kRadix = 256;
constexpr int kSortBlock = 256;  // one thread per digit in the per-tile digit work
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096 keys per tile
constexpr uint32_t kFlagAgg = 1u << 30, kFlagInc = 2u << 30, kValueMask = (1u << 30) - 1;
constexpr uint32_t kLookbackPolls = 1u << 22;  // default poll limit of one tile's look-back
#ifndef CPT_LOOKBACK_WINDOW
#define CPT_LOOKBACK_WINDOW 4
#endif
constexpr int kLookbackWindow = CPT_LOOKBACK_WINDOW;  // predecessor words read per look-back round

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

// Where a pass takes its (key, value) pairs from.
//   kSrcKeys    key = kin[i], value = vin[i]
//   kSrcIndex   key = kin[i], value = i (the first pass)
//   kSrcLow64   key = low 32 bits of g64[i], value = i (the first pass over 64-bit keys
//               sorted as two 32-bit halves)
//   kSrcHigh64  value = vin[i], key = high 32 bits of g64[value]
//   kSrcFull64  value = vin[i], key = g64[value] (the last pass: whole keys written out)
// A 64-bit key sorted by its low half (4 stable passes) and then by its high half (4
// stable passes) ends in the order of 8 stable passes over the whole key; the 32-bit
// passes move 8 B per element instead of 12 and, with half the staging memory, keep
// more tiles in flight per SM.
enum : int { kSrcKeys = 0, kSrcIndex = 1, kSrcLow64 = 2, kSrcHigh64 = 3, kSrcFull64 = 4 };

#ifndef CPT_SORT32_MIN_BLOCKS
#define CPT_SORT32_MIN_BLOCKS 3  // 80 registers, no spills (four tiles per SM at 64 registers spill: 0.62 vs 0.59 ms per 5.2 M-key sort)
#endif
template <typename K>
constexpr int onesweep_min_blocks() { return sizeof(K) == 4 ? CPT_SORT32_MIN_BLOCKS : 3; }

// One digit pass. Tiles are claimed in launch order through tile_counter, so a
// tile only ever waits on tiles already owned by running blocks (which publish
// their own counts before they wait): the look-back always completes; the poll
// bound (wait.poll_limit polls of one tile, then CPT_STATUS_TIMEOUT and the tile
// goes on with the prefix it has) is a guard, not a scheduling assumption. Within
// the pass that timed out, output positions stay inside [0, n), because a prefix read
// from the look-back never exceeds the true one. Its output is no longer a
// permutation, though (positions written twice, others left with whatever the buffer
// held), so a later pass over it would count digits the global histogram does not
// hold and could scatter past n: every pass therefore checks the status word when a
// block starts (one read, shared by the block) and returns at once after a timeout,
// like the kernels that follow the sort. A gathered value is clamped into [0, n)
// before it indexes g64 all the same.
template <typename K, int kSrc>
__device__ __forceinline__ void onesweep_pass(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                              const uint64_t* __restrict__ g64, K* __restrict__ kout,
                                              uint32_t* __restrict__ vout, uint32_t n_arg,
                                              const uint32_t* __restrict__ n_ptr, int shift,
                                              const uint32_t* __restrict__ offsets, uint32_t* __restrict__ lookback,
                                              uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status,
                                              SortWait wait)
{
    static_assert(kSrc == kSrcKeys || kSrc == kSrcIndex || sizeof(K) == (kSrc == kSrcFull64 ? 8 : 4),
                  "64-bit sources give 32-bit halves or whole 64-bit keys");
    extern __shared__ __align__(16) unsigned char smem[];
    K* s_keys = reinterpret_cast<K*>(smem);
    uint32_t* s_vals = reinterpret_cast<uint32_t*>(s_keys + kSortTile);
    uint32_t* s_hist = s_vals + kSortTile;       // [warp][digit]
    uint32_t* s_off = s_hist + kSortWarps * kRadix;  // tile-local exclusive offset per digit
    uint32_t* s_base = s_off + kRadix;           // global output base per digit
    __shared__ uint32_t s_tile, s_stop;
    __shared__ uint32_t s_wsum[kSortWarps];

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_stop = status ? (__ldcg(status) & CPT_STATUS_TIMEOUT) : 0u;
        s_tile = s_stop ? 0u : atomicAdd(tile_counter, 1u);
    }
    for (uint32_t i = tid; i < kSortWarps * kRadix; i += kSortBlock) s_hist[i] = 0;
    __syncthreads();
    if (s_stop) return;  // an earlier wait ran out: this sort's result is void (uniform per block)
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
        const uint32_t idx = wbase + k * 32 + lane;
        const bool valid = idx < n;
        if (kSrc == kSrcKeys || kSrc == kSrcIndex) {
            key[k] = valid ? kin[idx] : (K)0;
            val[k] = kSrc == kSrcIndex ? idx : (valid ? vin[idx] : 0u);
        } else if (kSrc == kSrcLow64) {
            key[k] = valid ? (K)(uint32_t)g64[idx] : (K)0;
            val[k] = idx;
        } else {
            val[k] = valid ? vin[idx] : 0u;
        }
    }
    if (kSrc == kSrcHigh64 || kSrc == kSrcFull64) {
#pragma unroll
        for (int k = 0; k < kSortItems; ++k) {
            const uint32_t idx = wbase + k * 32 + lane;
            const uint64_t w = idx < n ? g64[val[k] < n ? val[k] : 0u] : 0ull;
            key[k] = kSrc == kSrcHigh64 ? (K)(uint32_t)(w >> 32) : (K)w;
        }
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

    // Decoupled look-back over the preceding tiles for this digit, kLookbackWindow
    // predecessors per round: their words are read together, then taken in order up to
    // the first inclusive one (done) or the first not yet published (polled again).
    uint32_t prefix = 0;
    if (tile > 0) {
        int j = (int)tile - 1;
        uint32_t polls = 0;
        bool timed_out = false, done = false;
        while (!done) {
            uint32_t v[kLookbackWindow];
#pragma unroll
            for (int q = 0; q < kLookbackWindow; ++q)
                v[q] = j - q >= 0 ? ld_volatile(&lookback[(size_t)(j - q) * kRadix + tid]) : 0u;
            int taken = 0;
            bool blocked = false;
#pragma unroll
            for (int q = 0; q < kLookbackWindow; ++q) {
                if (done || blocked) continue;
                const uint32_t f = v[q] & ~kValueMask;
                if (f == 0) { blocked = true; continue; }
                prefix += v[q] & kValueMask;
                ++taken;
                if (f == kFlagInc) done = true;
            }
            j -= taken;
            if (done) break;
            if (taken == 0) {
                if (++polls > wait.poll_limit) { timed_out = true; break; }
                if (polls > 32) __nanosleep(100);
            }
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

#ifndef CPT_SORT_MIN_BLOCKS
#define CPT_SORT_MIN_BLOCKS 3  // 80 registers: three 4096-key tiles per SM (0.63 vs 0.67 ms per 5.2 M-key sort)
#endif

// One digit pass over (key, value) pairs; kFirst: the values are the element indices.
template <typename K, bool kFirst>
__global__ void __launch_bounds__(kSortBlock, CPT_SORT_MIN_BLOCKS) k_onesweep(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                         K* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n_arg,
                                                         const uint32_t* __restrict__ n_ptr,
                                                         int shift, const uint32_t* __restrict__ offsets,
                                                         uint32_t* __restrict__ lookback,
                                                         uint32_t* __restrict__ tile_counter,
                                                         uint32_t* __restrict__ status, SortWait wait = SortWait())
{
    onesweep_pass<K, kFirst ? kSrcIndex : kSrcKeys>(kin, vin, nullptr, kout, vout, n_arg, n_ptr, shift, offsets,
                                                    lookback, tile_counter, status, wait);
}

// One digit pass of a 64-bit key sort done as two 32-bit halves (kSrcLow64,
// kSrcKeys over the halves, kSrcHigh64, kSrcFull64).
template <typename K, int kSrc>
__global__ void __launch_bounds__(kSortBlock, onesweep_min_blocks<K>()) k_onesweep_halves(
    const K* __restrict__ kin, const uint32_t* __restrict__ vin, const uint64_t* __restrict__ g64,
    K* __restrict__ kout, uint32_t* __restrict__ vout, uint32_t n_arg, const uint32_t* __restrict__ n_ptr,
    int shift, const uint32_t* __restrict__ offsets, uint32_t* __restrict__ lookback,
    uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status, SortWait wait)
{
    onesweep_pass<K, kSrc>(kin, vin, g64, kout, vout, n_arg, n_ptr, shift, offsets, lookback, tile_counter, status,
                           wait);
}

// The 8 passes of a stable sort of 64-bit keys as 32-bit halves, with values that
// start as the element indices. keys_in (input order) stays intact: the gathers read
// it. The halves ping-pong in the two halves of keys_out (2 x cap words, unused until
// the last pass), which the last pass fills with the sorted whole keys when
// whole_keys is set (otherwise it is one more 32-bit pass and only the order is the
// result); pass p writes vals[p & 1], so the order ends in vals[1]. The element count
// is n, or *n_ptr on the device (cap bounds it and sizes the grids). offsets: the
// 8 x 256 digit offsets; lookback: 8 regions of tiles x 256 words, tile_counters: 8
// words, all zeroed. prof: each pass timed as K_ONESWEEP.
inline int onesweep_sort64_halves(const uint64_t* keys_in, uint64_t* keys_out, uint32_t cap, uint32_t n,
                                  const uint32_t* n_ptr, uint32_t* const vals[2], const uint32_t* offsets,
                                  uint32_t* lookback, uint32_t* tile_counters, uint32_t* status, SortWait wait,
                                  bool whole_keys, bool prof, cudaStream_t stream)
{
    constexpr int P = 8;
    const uint32_t tiles = (cap + kSortTile - 1) / kSortTile;
    const size_t smem32 = onesweep_smem<uint32_t>(), smem64 = onesweep_smem<uint64_t>();
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep_halves<uint32_t, kSrcLow64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep_halves<uint32_t, kSrcKeys>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep_halves<uint32_t, kSrcHigh64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep_halves<uint64_t, kSrcFull64>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem64));
    uint32_t* half[2] = {reinterpret_cast<uint32_t*>(keys_out), reinterpret_cast<uint32_t*>(keys_out) + cap};
    for (int p = 0; p < P; ++p) {
        const uint32_t* vin = vals[(p + 1) & 1];
        uint32_t* vout = vals[p & 1];
        uint32_t* lb = lookback + (size_t)p * tiles * kRadix;
        const uint32_t* off = offsets + p * kRadix;
        SortWait w = wait;
        if (p) w.withhold_tile0 = 0;  // (the test hook stalls the first pass only)
        auto launch = [&]() {
            if (p == 0)
                k_onesweep_halves<uint32_t, kSrcLow64><<<tiles, kSortBlock, smem32, stream>>>(
                    nullptr, nullptr, keys_in, half[0], vout, n, n_ptr, 0, off, lb, tile_counters + p, status, w);
            else if (p == 4)
                k_onesweep_halves<uint32_t, kSrcHigh64><<<tiles, kSortBlock, smem32, stream>>>(
                    nullptr, vin, keys_in, half[0], vout, n, n_ptr, 0, off, lb, tile_counters + p, status, w);
            else if (p == P - 1 && whole_keys)
                k_onesweep_halves<uint64_t, kSrcFull64><<<tiles, kSortBlock, smem64, stream>>>(
                    nullptr, vin, keys_in, keys_out, vout, n, n_ptr, 8 * p, off, lb, tile_counters + p, status, w);
            else
                k_onesweep_halves<uint32_t, kSrcKeys><<<tiles, kSortBlock, smem32, stream>>>(
                    half[(p + 1) & 1], vin, nullptr, half[p & 1], vout, n, n_ptr, 8 * (p & 3), off, lb,
                    tile_counters + p, status, w);
        };
        if (prof) {
            ProfScope ps(K_ONESWEEP, stream);
            launch();
        } else {
            launch();
        }
        CPT_LAUNCH_CHECK();
    }
    return CPT_OK;
}


}  // namespace cpt
