// LBVH construction for sm_100a: Morton codes, onesweep radix sort, Karras
// topology, atomic bottom-up refit.
//
// Replaces CUDA::BVHBuilder::build (source/application/cuda/BVHBuilder.cu:207-269)
// and its four thrust passes. Outputs are the reference's arrays, bit for bit,
// plus the compact traversal records used by trace.cu / render.cu:
//
//   kernel             reference                               reads / writes per triangle
//   k_bounds*          caller's enclosingBBox (PathTracingApp.cpp:113), optional
//   k_morton           morton_encoder (BVHBuilder.cu:12-32)    40 B tri -> K B key, digit histograms
//   k_scan_offsets     (part of thrust::sort_by_key)           P x 256 counters
//   k_onesweep x P     thrust::sort_by_key (BVHBuilder.cu:234) K+4 B in, K+4 B out per pass
//   k_topology         radix_tree_construction_kernel (:107-201) keys -> Node, parents
//   k_gather_refit     compute_internal_node_bbox_kernel (:39-98) + the triangle permutation
//                      + the 96-B traversal nodes (child slots filled bottom-up)
//
// The sort is a least-significant-digit radix sort with 8-bit digits in the
// onesweep form (one global histogram pass, then one pass per digit in which each
// tile ranks its keys with warp-level match/popc scans and finds its output base
// by decoupled look-back over the preceding tiles). LSD radix sorting is stable,
// which reproduces thrust's stable sort_by_key order for equal keys. The
// look-back wait is bounded: after its poll limit (kLookbackPolls, or the
// caller's CPT_BUILD_LOOKBACK_LIMIT) it records CPT_STATUS_TIMEOUT and proceeds,
// so no launch can hang; topology and refit then return at once, and the parent
// walk of the refit is bounded by n - 1 steps.
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"
#include "onesweep.cuh"
#include "lbvh_common.cuh"

namespace cpt {

constexpr int kMortonBlock = 256;
constexpr int kBoundsBlock = 320;   // 10 warps; a multiple of 5 (one word phase per thread)
constexpr int kBoundsBlocks = 888;  // 148 SMs x 6 blocks

struct BoxArg {
    float mn[3];
    float inv[3];
    const float* dev;  // device box (min, max) when the host gave none
};

// ---------------------------------------------------------------------------
// Enclosing box on the device (when the caller passes none): per-block partial
// boxes, then one block folds them in a fixed order.
// ---------------------------------------------------------------------------
// The soup is read as one flat array of 16-B words (n x 10 floats, 16-B aligned): a
// float at flat position f belongs to field f % 10 of its triangle, a coordinate of
// axis (f % 10) % 3 when f % 10 < 9 (the tenth is info_idx). Coalesced 16-B loads
// instead of nine 4-B loads 40 B apart per triangle. Word q starts at field
// (4 q) % 10, which depends on q % 5 only; with a block of 320 threads (a multiple of
// 5) and a grid-stride loop every word a thread reads has the same phase
// threadIdx.x % 5, so each of the four lanes of the word keeps its own running
// min / max in registers and is mapped to its axis once, after the loop.
__device__ __forceinline__ void bounds_fold(float lo, float hi, uint32_t field, float mn[3], float mx[3])
{
#pragma unroll
    for (uint32_t a = 0; a < 3; ++a) {
        const bool take = field < 9u && field % 3u == a;
        mn[a] = take ? gmin(mn[a], lo) : mn[a];
        mx[a] = take ? gmax(mx[a], hi) : mx[a];
    }
}

__global__ void __launch_bounds__(kBoundsBlock) k_bounds_partial(const float* __restrict__ tris, uint32_t n,
                                                                 float* __restrict__ partial)
{
    static_assert(kBoundsBlock % 5 == 0 && kBoundsBlock % 32 == 0, "one phase per thread, whole warps");
    float lo[4] = {FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX}, hi[4] = {-FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    const uint64_t floats = 10ull * n, quads = floats / 4;
    const float4* q4 = reinterpret_cast<const float4*>(tris);
    for (uint64_t q = (uint64_t)blockIdx.x * kBoundsBlock + threadIdx.x; q < quads;
         q += (uint64_t)gridDim.x * kBoundsBlock) {
        const float4 v = __ldg(q4 + q);
        lo[0] = gmin(lo[0], v.x); hi[0] = gmax(hi[0], v.x);
        lo[1] = gmin(lo[1], v.y); hi[1] = gmax(hi[1], v.y);
        lo[2] = gmin(lo[2], v.z); hi[2] = gmax(hi[2], v.z);
        lo[3] = gmin(lo[3], v.w); hi[3] = gmax(hi[3], v.w);
    }
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    const uint32_t f0 = (4u * (threadIdx.x % 5u)) % 10u;
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) bounds_fold(lo[j], hi[j], (f0 + j) % 10u, mn, mx);
    if (blockIdx.x == 0 && threadIdx.x < floats - 4 * quads) {  // an odd count leaves fields 8 and 9 of the last
        const float v = tris[4 * quads + threadIdx.x];
        bounds_fold(v, v, 8u + threadIdx.x, mn, mx);
    }
    // Block fold: warp shuffles, then one value per warp through shared memory.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            mn[a] = gmin(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = gmax(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    constexpr int kWarps = kBoundsBlock / 32;
    __shared__ float s[6][kWarps];
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 3; ++a) { s[a][threadIdx.x >> 5] = mn[a]; s[3 + a][threadIdx.x >> 5] = mx[a]; }
    __syncthreads();
    if (threadIdx.x < 6) {
        float b = s[threadIdx.x][0];
        for (int w = 1; w < kWarps; ++w) b = threadIdx.x < 3 ? gmin(b, s[threadIdx.x][w]) : gmax(b, s[threadIdx.x][w]);
        partial[6 * blockIdx.x + threadIdx.x] = b;
    }
}

// One block folds the per-block boxes: each thread a strided subset, then shuffles.
__global__ void __launch_bounds__(256) k_bounds_final(const float* __restrict__ partial, int blocks,
                                                      float* __restrict__ box)
{
    float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = threadIdx.x; i < blocks; i += blockDim.x)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b[a] = gmin(b[a], partial[6 * i + a]);
            b[3 + a] = gmax(b[3 + a], partial[6 * i + 3 + a]);
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            b[a] = gmin(b[a], __shfl_xor_sync(0xffffffffu, b[a], o));
            b[3 + a] = gmax(b[3 + a], __shfl_xor_sync(0xffffffffu, b[3 + a], o));
        }
    __shared__ float s[6][8];
    if ((threadIdx.x & 31) == 0)
        for (int a = 0; a < 6; ++a) s[a][threadIdx.x >> 5] = b[a];
    __syncthreads();
    if (threadIdx.x < 6) {
        const int warps = (int)(blockDim.x + 31) / 32;
        float r = s[threadIdx.x][0];
        for (int w = 1; w < warps; ++w) r = threadIdx.x < 3 ? gmin(r, s[threadIdx.x][w]) : gmax(r, s[threadIdx.x][w]);
        box[threadIdx.x] = r;
    }
}

// ---------------------------------------------------------------------------
// Morton codes + per-pass digit histograms + zeroing of the sort's look-back
// state. One key per triangle: centroid (v0 + v1 + v2) / 3 quantized to
// 2^order cells per axis of the enclosing box (BVHBuilder.cu:19-28).
// ---------------------------------------------------------------------------
template <typename K>
__global__ void __launch_bounds__(kMortonBlock) k_morton(const float* __restrict__ tris, uint32_t n, BoxArg box,
                                                         K* __restrict__ keys, uint32_t* __restrict__ hist,
                                                         uint32_t* __restrict__ zero, size_t zero_words,
                                                         uint32_t* __restrict__ status)
{
    constexpr int P = KeyTraits<K>::passes;
    constexpr int order = KeyTraits<K>::order;
    __shared__ uint32_t s_hist[P * kRadix];
    __shared__ float s_box[6];
    for (int i = threadIdx.x; i < P * kRadix; i += blockDim.x) s_hist[i] = 0;
    if (threadIdx.x < 3) {
        if (box.dev) {
            float mn = box.dev[threadIdx.x], mx = box.dev[3 + threadIdx.x];
            s_box[threadIdx.x] = mn;
            s_box[3 + threadIdx.x] = __frcp_rn(__fsub_rn(mx, mn));  // 1.0f / scale (BVHBuilder.cu:17)
        } else {
            s_box[threadIdx.x] = box.mn[threadIdx.x];
            s_box[3 + threadIdx.x] = box.inv[threadIdx.x];
        }
    }
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t gsize = (size_t)gridDim.x * blockDim.x;
    for (size_t i = gtid; i < zero_words; i += gsize) zero[i] = 0;
    __syncthreads();
    const uint32_t cells = 1u << order;
    uint32_t bad = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float2* t2 = reinterpret_cast<const float2*>(tris + 10ull * i);
        float2 a = __ldg(t2), b = __ldg(t2 + 1), c = __ldg(t2 + 2), d = __ldg(t2 + 3), e = __ldg(t2 + 4);
        float v[9] = {a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x};
#pragma unroll
        for (int j = 0; j < 9; ++j) bad |= !isfinite(v[j]);
        uint32_t q[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            float cen = __fdiv_rn(__fadd_rn(__fadd_rn(v[ax], v[3 + ax]), v[6 + ax]), 3.0f);
            q[ax] = quantize(__fmul_rn(__fsub_rn(cen, s_box[ax]), s_box[3 + ax]), cells);
        }
        uint64_t k = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        keys[i] = (K)k;
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(&s_hist[p * kRadix + (uint32_t)((k >> (8 * p)) & 0xFF)], 1u);
    }
    if (bad) atomicOr(status, CPT_STATUS_NONFINITE);
    __syncthreads();
    for (int i = threadIdx.x; i < P * kRadix; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// ---------------------------------------------------------------------------
// Karras radix tree: k_topology (lbvh_common.cuh).
// ---------------------------------------------------------------------------
// Triangle permutation fused with the bottom-up refit. Thread i gathers sorted
// triangle i (the 40-B reference record), computes its leaf box, then walks up.
// At each parent it writes its child slot of the parent's 96-B traversal node
// (the triangle for a leaf, the box for an internal node); the second child to
// arrive (atomic counter) reads its sibling's box — the box the sibling's thread
// computed, which for a leaf is the reference's box of the triangle's vertices
// (BVHBuilder.cu:73-80) — and stores left.unite(right). Below the nodes whose leaf
// range leaves the block, the counter and the sibling's box live in shared memory
// (block-scope fences order them); above, the counter increment is a global
// acquire-release atomic: it publishes this thread's slot and box stores and makes the
// sibling's visible to the second arriver (the reference's refit has no ordering
// between them, BVHBuilder.cu:63-86).
// ---------------------------------------------------------------------------
#ifndef CPT_REFIT_BLOCK
#define CPT_REFIT_BLOCK 64
#endif
// leaves per block: the nodes below them arrive in shared memory (C5 refit, 16.8 M
// triangles: 1.67 / 1.70 / 1.77 / 2.01 ms at 64 / 128 / 256 / 512; 2.22 ms all global)
constexpr int kRefitBlock = CPT_REFIT_BLOCK;

// A climbing thread arrives at node p and learns whether it is the second child to
// arrive (and may go on). Nodes whose leaf range lies inside this block's leaves have
// both children completed by threads of this block: they use a shared-memory counter,
// and the first arriver leaves its box in shared memory for the second. Other nodes
// use the global counter with acquire-release order, the sibling's box coming from the
// node-box array (or, for a leaf sibling, its sorted triangle).
__global__ void __launch_bounds__(kRefitBlock) k_gather_refit(const float* __restrict__ tris_in, const uint32_t* __restrict__ order,
                                                      uint32_t n, float* __restrict__ tris_out,
                                                      const uint32_t* __restrict__ children,
                                                      const uint32_t* __restrict__ parents_leaf,
                                                      const uint32_t* __restrict__ parents_internal,
                                                      int* __restrict__ counters, float* __restrict__ nodes,
                                                      cpt_bbox* __restrict__ node_boxes, uint32_t* __restrict__ status)
{
    __shared__ int s_count[kRefitBlock];
    __shared__ float s_box[2 * kRefitBlock][6];  // [2 * (p - base) + side]: the first arriver's box
    const uint32_t base = blockIdx.x * kRefitBlock;
    s_count[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = base + threadIdx.x;
    if (i >= n) return;
    if (sort_timed_out(status)) return;  // the order is not a sort: nothing to gather or refit
    (void)children;
    gather_refit_leaf(tris_in, order[i], i, n, base, min(n, base + (uint32_t)kRefitBlock), tris_out, parents_leaf,
                      parents_internal, counters, nodes, node_boxes, status, s_count, s_box);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename K>
struct SortScratch {
    K* keys_alt;
    uint32_t* vals[2];
    uint32_t* hist;
    uint32_t* offsets;
    uint32_t* zero_region;  // tile counters + look-back, zeroed by k_morton
    size_t zero_words;
    uint32_t* tile_counters;
    uint32_t* lookback;
    int* counters;
    float* bounds_partial;
    float* dev_box;
    float* tris_copy;
};

inline uint32_t num_tiles(uint32_t n) { return (n + kSortTile - 1) / kSortTile; }

template <typename K>
size_t scratch_layout(uint32_t n, void* base, SortScratch<K>* s)
{
    constexpr int P = KeyTraits<K>::passes;
    Carver c(base);
    SortScratch<K> t;
    t.keys_alt = c.take<K>(n);
    t.vals[0] = c.take<uint32_t>(n);
    t.vals[1] = c.take<uint32_t>(n);
    t.hist = c.take<uint32_t>((size_t)P * kRadix);
    t.offsets = c.take<uint32_t>((size_t)P * kRadix);
    t.zero_words = 32 + (size_t)P * num_tiles(n) * kRadix;
    t.zero_region = c.take<uint32_t>(t.zero_words);
    t.tile_counters = t.zero_region;
    t.lookback = t.zero_region ? t.zero_region + 32 : nullptr;
    t.counters = c.take<int>(n);
    t.bounds_partial = c.take<float>(6 * kBoundsBlocks);
    t.dev_box = c.take<float>(8);
    t.tris_copy = c.take<float>(10ull * n);
    if (s) *s = t;
    return c.used();
}

// The stable key sort: P passes of 8-bit digits. 32-bit keys: key and value passes
// ping-pong between keys and keys_alt. 64-bit keys (in keys_alt, input order): four
// passes over the low halves and three over the high halves, ping-ponging 32-bit
// halves in the two halves of `keys` (free until the last pass), then the last pass
// gathers whole keys by value and writes them, sorted, to `keys`. Values end in
// vals[(P - 1) & 1] either way.
template <typename K>
int sort_keys(const SortScratch<K>& s, uint32_t n, K* keys, uint32_t* status, SortWait wait, cudaStream_t stream)
{
    if constexpr (sizeof(K) == 8) {
        return onesweep_sort64_halves(reinterpret_cast<const uint64_t*>(s.keys_alt), reinterpret_cast<uint64_t*>(keys),
                                      n, n, nullptr, s.vals, s.offsets, s.lookback, s.tile_counters, status, wait, true,
                                      true, stream);
    } else {
        constexpr int P = KeyTraits<K>::passes;
        const uint32_t tiles = num_tiles(n);
        const size_t smem = onesweep_smem<K>();
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        K* kbuf[2] = {keys, s.keys_alt};
        for (int p = 0; p < P; ++p) {
            const K* kin = kbuf[p & 1];
            K* kout = kbuf[(p + 1) & 1];
            const uint32_t* vin = p == 0 ? nullptr : s.vals[(p + 1) & 1];
            uint32_t* vout = s.vals[p & 1];
            uint32_t* lb = s.lookback + (size_t)p * tiles * kRadix;
            CPT_PROF(K_ONESWEEP, stream);
            if (p == 0)
                k_onesweep<K, true><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, n, nullptr, 8 * p,
                                                                         s.offsets + p * kRadix,
                                                                         lb, s.tile_counters + p, status, wait);
            else {
                SortWait later = wait;
                later.withhold_tile0 = 0;  // (the test hook stalls the first pass only)
                k_onesweep<K, false><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, n, nullptr, 8 * p,
                                                                          s.offsets + p * kRadix,
                                                                          lb, s.tile_counters + p, status, later);
            }
            CPT_LAUNCH_CHECK();
        }
        return CPT_OK;
    }
}

template <typename K>
int build_impl(const cpt_triangle* tris_in, uint32_t n, const float* host_box, cpt_bvh* bvh, void* scratch,
               SortWait wait, cudaStream_t stream)
{
    constexpr int P = KeyTraits<K>::passes;
    SortScratch<K> s;
    scratch_layout<K>(n, scratch, &s);
    const float* tri_src = reinterpret_cast<const float*>(tris_in);
    if (tris_in == bvh->tris) {
        // In-place build (the reference permutes DeviceSceneDescription::triangles):
        // gather from a copy.
        CPT_CUDA_TRY(cudaMemcpyAsync(s.tris_copy, tris_in, sizeof(cpt_triangle) * (size_t)n, cudaMemcpyDeviceToDevice, stream));
        tri_src = s.tris_copy;
    }
    CPT_CUDA_TRY(cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * P * kRadix, stream));
    CPT_CUDA_TRY(cudaMemsetAsync(bvh->status, 0, 4 * sizeof(uint32_t), stream));

    BoxArg box{};
    if (host_box) {
        for (int a = 0; a < 3; ++a) {
            box.mn[a] = host_box[a];
            box.inv[a] = 1.0f / (host_box[3 + a] - host_box[a]);
        }
        box.dev = nullptr;
    } else {
        {
            CPT_PROF(K_BOUNDS, stream);
            k_bounds_partial<<<kBoundsBlocks, kBoundsBlock, 0, stream>>>(tri_src, n, s.bounds_partial);
        }
        CPT_LAUNCH_CHECK();
        {
            CPT_PROF(K_BOUNDS, stream);
            k_bounds_final<<<1, 256, 0, stream>>>(s.bounds_partial, kBoundsBlocks, s.dev_box);
        }
        CPT_LAUNCH_CHECK();
        box.dev = s.dev_box;
    }

    K* keys = static_cast<K*>(bvh->keys);
    const int sms = sm_count();
    const int morton_blocks = (int)std::min<size_t>((n + kMortonBlock - 1) / kMortonBlock, (size_t)sms * 8);
    {
        CPT_PROF(K_MORTON, stream);
        // 64-bit keys go to keys_alt: the sort reads them from there (sort_keys)
        k_morton<K><<<morton_blocks, kMortonBlock, 0, stream>>>(tri_src, n, box, sizeof(K) == 8 ? s.keys_alt : keys,
                                                                s.hist, s.zero_region, s.zero_words, bvh->status);
    }
    CPT_LAUNCH_CHECK();
    {
        CPT_PROF(K_SCAN, stream);
        k_scan_offsets<<<P, kRadix, 0, stream>>>(s.hist, s.offsets);
    }
    CPT_LAUNCH_CHECK();

    if (const int rc = sort_keys<K>(s, n, keys, bvh->status, wait, stream)) return rc;
    // P is even: keys end in bvh->keys, values in vals[(P - 1) & 1].
    const uint32_t* order = s.vals[(P - 1) & 1];

    const uint32_t inner = n - 1;
    {
        CPT_PROF(K_TOPOLOGY, stream);
        k_topology<K><<<(inner + 255) / 256, 256, 0, stream>>>(keys, n, nullptr, bvh->children, bvh->parents_leaf,
                                                                bvh->parents_internal, s.counters,
                                                                static_cast<float4*>(bvh->nodes), bvh->status,
                                                                inner);
    }
    CPT_LAUNCH_CHECK();
    {
        CPT_PROF(K_GATHER_REFIT, stream);
        k_gather_refit<<<(n + kRefitBlock - 1) / kRefitBlock, kRefitBlock, 0, stream>>>(tri_src, order, n, reinterpret_cast<float*>(bvh->tris),
                                                             bvh->children, bvh->parents_leaf, bvh->parents_internal,
                                                             s.counters, static_cast<float*>(bvh->nodes),
                                                             bvh->node_boxes, bvh->status);
    }
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

inline size_t key_bytes(int bits) { return bits == 30 ? 4 : 8; }

}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_bvh_bytes(uint32_t n, int morton_bits)
{
    if (n < 2 || (morton_bits != 30 && morton_bits != 63)) return 0;
    Carver c(nullptr);
    c.take<cpt_triangle>(n);
    c.take<char>(key_bytes(morton_bits) * n);
    c.take<uint32_t>(n - 1);
    c.take<uint32_t>(n);
    c.take<uint32_t>(n - 1);
    c.take<cpt_bbox>(n - 1);
    c.take<float4>(6ull * (n - 1));
    c.take<uint32_t>(4);
    return c.used();
}

extern "C" int cpt_bvh_bind(void* mem, size_t bytes, uint32_t n, int morton_bits, cpt_bvh* out)
{
    if (!mem || !out || n < 2 || n > kMaxTriangles || (morton_bits != 30 && morton_bits != 63))
        return CPT_ERR_INVALID_ARGUMENT;
    if (bytes < cpt_bvh_bytes(n, morton_bits)) return CPT_ERR_SCRATCH_TOO_SMALL;
    Carver c(mem);
    out->n = n;
    out->morton_bits = morton_bits;
    out->tris = c.take<cpt_triangle>(n);
    out->keys = c.take<char>(key_bytes(morton_bits) * n);
    out->children = c.take<uint32_t>(n - 1);
    out->parents_leaf = c.take<uint32_t>(n);
    out->parents_internal = c.take<uint32_t>(n - 1);
    out->node_boxes = c.take<cpt_bbox>(n - 1);
    out->nodes = c.take<float4>(6ull * (n - 1));
    out->status = c.take<uint32_t>(4);
    out->split_nodes = nullptr;
    out->split_capacity = 0;
    out->wide_nodes = nullptr;
    out->wide_tris = nullptr;
    out->wide_capacity = 0;
    return CPT_OK;
}

extern "C" size_t cpt_lbvh_scratch_bytes(uint32_t n, int morton_bits)
{
    if (n < 2 || n > kMaxTriangles) return 0;
    if (morton_bits == 30) return scratch_layout<uint32_t>(n, nullptr, nullptr);
    if (morton_bits == 63) return scratch_layout<uint64_t>(n, nullptr, nullptr);
    return 0;
}

extern "C" int cpt_status_check(const uint32_t* d_status, cudaStream_t stream)
{
    if (!d_status) return CPT_ERR_INVALID_ARGUMENT;
    uint32_t h[4] = {0, 0, 0, 0};
    CPT_CUDA_TRY(cudaMemcpyAsync(h, d_status, sizeof(h), cudaMemcpyDeviceToHost, stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h[0] & CPT_STATUS_NONFINITE) return CPT_ERR_NONFINITE_INPUT;
    if (h[0] & CPT_STATUS_TIMEOUT) return CPT_ERR_DEVICE_TIMEOUT;
    if (h[0] & CPT_STATUS_STACK_OVERFLOW) return CPT_ERR_STACK_OVERFLOW;
    if (h[0] & CPT_STATUS_BAD_INDEX) return CPT_ERR_BAD_INDEX;
    return CPT_OK;
}

extern "C" int cpt_lbvh_build(const cpt_triangle* tris_in, uint32_t n, const float* enclosing_box, int morton_bits,
                              cpt_bvh* bvh, void* scratch, size_t scratch_bytes, uint32_t flags, cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_build");
    if (bvh) {  // split and wide trees of the previous build are stale
        bvh->split_nodes = nullptr;
        bvh->split_capacity = 0;
        bvh->wide_nodes = nullptr;
        bvh->wide_tris = nullptr;
        bvh->wide_capacity = 0;
    }
    if (!tris_in || !bvh || !scratch || n < 2 || n > kMaxTriangles) return CPT_ERR_INVALID_ARGUMENT;
    if (morton_bits != 30 && morton_bits != 63) return CPT_ERR_INVALID_ARGUMENT;
    if (bvh->n != n || bvh->morton_bits != morton_bits || !bvh->tris || !bvh->keys || !bvh->children ||
        !bvh->parents_leaf || !bvh->parents_internal || !bvh->node_boxes || !bvh->nodes || !bvh->status)
        return CPT_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(tris_in) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 255) ||
        (reinterpret_cast<uintptr_t>(bvh->nodes) & 15) || (reinterpret_cast<uintptr_t>(bvh->tris) & 15))
        return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < cpt_lbvh_scratch_bytes(n, morton_bits)) return CPT_ERR_SCRATCH_TOO_SMALL;
    if (flags & ~(CPT_BUILD_CHECK | CPT_BUILD_TEST_WITHHOLD | CPT_BUILD_LOOKBACK_LIMIT(31)))
        return CPT_ERR_INVALID_ARGUMENT;
    SortWait wait;
    const uint32_t log2_polls = (flags >> 8) & 31u;
    if (log2_polls) wait.poll_limit = 1u << log2_polls;
    if (flags & CPT_BUILD_TEST_WITHHOLD) {
        // the stalled wait must be short: an explicit limit of at most 2^16 polls
        if (log2_polls == 0 || log2_polls > 16) return CPT_ERR_INVALID_ARGUMENT;
        wait.withhold_tile0 = 1;
    }
    int rc = morton_bits == 30 ? build_impl<uint32_t>(tris_in, n, enclosing_box, bvh, scratch, wait, stream)
                               : build_impl<uint64_t>(tris_in, n, enclosing_box, bvh, scratch, wait, stream);
    if (rc != CPT_OK || !(flags & CPT_BUILD_CHECK)) return rc;
    rc = cpt_status_check(bvh->status, stream);
    if (rc != CPT_OK) return rc;
    // Root-volume self-check of BVHBuilder.cu:258-265 (absolute epsilon 1e-7,
    // source/engine/util/math.h:22,68), against the host box or the device box.
    cpt_bbox root;
    CPT_CUDA_TRY(cudaMemcpyAsync(&root, bvh->node_boxes, sizeof(root), cudaMemcpyDeviceToHost, stream));
    float eb[6];
    if (enclosing_box) {
        for (int a = 0; a < 6; ++a) eb[a] = enclosing_box[a];
    } else {
        SortScratch<uint32_t> s32;
        SortScratch<uint64_t> s64;
        const float* dev_box = morton_bits == 30 ? (scratch_layout<uint32_t>(n, scratch, &s32), s32.dev_box)
                                                 : (scratch_layout<uint64_t>(n, scratch, &s64), s64.dev_box);
        CPT_CUDA_TRY(cudaMemcpyAsync(eb, dev_box, sizeof(eb), cudaMemcpyDeviceToHost, stream));
    }
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    float ve = (eb[3] - eb[0]) * (eb[4] - eb[1]) * (eb[5] - eb[2]);
    float vr = (root.max[0] - root.min[0]) * (root.max[1] - root.min[1]) * (root.max[2] - root.min[2]);
    if (!(fabsf(ve - vr) <= 1e-7f)) return CPT_ERR_CHECK_FAILED;
    return CPT_OK;
}
