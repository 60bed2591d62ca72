// Batched LBVH build: the LBVHs of many scenes (triangle soups of any sizes) in one
// fixed sequence of launches, each covering every scene.
//
// The reference builds one scene per call (CUDA::BVHBuilder::build,
// source/application/cuda/BVHBuilder.cu:207-269), as cpt_lbvh_build does; a batch of
// 64 small-to-medium scenes then costs 64 launch sequences, most of them far too
// small to fill the GPU. Here the scenes are segments of one index space
// [0, N_total): scene s holds global indices [off_s, off_s + n_s).
//
//   k_batch_morton      every triangle's key in its scene's box; digit histograms of
//                       the key passes and of the scene digit; per-scene status cleared
//   k_scan_offsets      as the single build, one block per pass
//   k_onesweep x P      the key passes over all scenes together (stable LSD)
//   k_batch_scene_ids   the scene of each element in key order
//   k_onesweep          one more stable pass on the scene id: order = (scene, key,
//                       input position), i.e. each scene's own stable key order
//   k_batch_keys        each scene's sorted keys, gathered into its output
//   k_batch_topology    Karras topology of every scene (one thread per internal node)
//   k_batch_refit       gather + bottom-up refit, blocks never straddling two scenes
//   k_batch_status      the batch's sort / input status copied into every scene's
//
// Every scene's outputs are those of cpt_lbvh_build on the same triangles and box,
// bit for bit: the same key arithmetic, the same stable order (ties by input
// position), the same topology and refit code (lbvh_common.cuh, lbvh.cu). The scene
// table travels by value as a kernel parameter, so a batch build records into a CUDA
// graph without host-side staging.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <mutex>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"
#include "onesweep.cuh"
#include "lbvh_common.cuh"

namespace cpt {

constexpr int kBatchRefitBlock = 64;  // leaves per refit block (as the single build's default)

namespace {

constexpr int kBatchBlock = 256;

struct BatchScene {
    const float* tris_in;   // the scene's input (or its copy in scratch for an in-place build)
    float* tris_out;        // bvh->tris
    void* keys;             // bvh->keys
    uint32_t* children;
    uint32_t* parents_leaf;
    uint32_t* parents_internal;
    cpt_bbox* node_boxes;
    float* nodes;
    uint32_t* status;
    float mn[3], inv[3];    // box minimum and 1 / extent, computed on the host as the single build
};

struct BatchTable {
    uint32_t scenes;
    uint32_t total;                              // N_total
    uint32_t off[CPT_MAX_BATCH_SCENES + 1];      // first global index of each scene
    uint32_t inner_off[CPT_MAX_BATCH_SCENES + 1];  // first global internal node (off - scene)
    uint32_t block_off[CPT_MAX_BATCH_SCENES + 1];  // first refit block
    BatchScene s[CPT_MAX_BATCH_SCENES];
};

// largest s with table[s] <= g (table ascending, table[0] = 0)
__device__ __forceinline__ uint32_t segment_of(const uint32_t* table, uint32_t count, uint32_t g)
{
    uint32_t lo = 0, hi = count;  // invariant: table[lo] <= g < table[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (table[mid] <= g) lo = mid; else hi = mid;
    }
    return lo;
}

template <typename K>
__global__ void __launch_bounds__(kBatchBlock) k_batch_morton(BatchTable bt, K* __restrict__ keys,
                                                              uint32_t* __restrict__ hist, uint32_t* __restrict__ zero,
                                                              size_t zero_words, uint32_t* __restrict__ batch_status)
{
    constexpr int P = KeyTraits<K>::passes;
    constexpr int order = KeyTraits<K>::order;
    __shared__ uint32_t s_hist[(P + 1) * kRadix];
    for (int i = threadIdx.x; i < (P + 1) * kRadix; i += blockDim.x) s_hist[i] = 0;
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t gsize = (size_t)gridDim.x * blockDim.x;
    for (size_t i = gtid; i < zero_words; i += gsize) zero[i] = 0;
    if (blockIdx.x == 0)  // each scene's status words start clear (later launches OR into them)
        for (uint32_t k = threadIdx.x; k < 4 * bt.scenes; k += blockDim.x) bt.s[k >> 2].status[k & 3] = 0;
    __syncthreads();
    const uint32_t cells = 1u << order;
    uint32_t bad = 0;
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.total; g += gridDim.x * blockDim.x) {
        const uint32_t sc = segment_of(bt.off, bt.scenes, g);
        const BatchScene& S = bt.s[sc];
        const float2* t2 = reinterpret_cast<const float2*>(S.tris_in + 10ull * (g - bt.off[sc]));
        const float2 a = __ldg(t2), b = __ldg(t2 + 1), c = __ldg(t2 + 2), d = __ldg(t2 + 3), e = __ldg(t2 + 4);
        const float v[9] = {a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x};
#pragma unroll
        for (int j = 0; j < 9; ++j) bad |= !isfinite(v[j]);
        uint32_t q[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {  // BVHBuilder.cu:19-28, as k_morton
            const float cen = __fdiv_rn(__fadd_rn(__fadd_rn(v[ax], v[3 + ax]), v[6 + ax]), 3.0f);
            q[ax] = quantize(__fmul_rn(__fsub_rn(cen, S.mn[ax]), S.inv[ax]), cells);
        }
        const uint64_t k = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
        keys[g] = (K)k;
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(&s_hist[p * kRadix + (uint32_t)((k >> (8 * p)) & 0xFF)], 1u);
        atomicAdd(&s_hist[P * kRadix + sc], 1u);
    }
    if (bad) atomicOr(batch_status, CPT_STATUS_NONFINITE);
    __syncthreads();
    for (int i = threadIdx.x; i < (P + 1) * kRadix; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// The scene of each element in the key-sorted order (values = global input index).
__global__ void __launch_bounds__(kBatchBlock) k_batch_scene_ids(BatchTable bt, const uint32_t* __restrict__ vals,
                                                                 uint32_t* __restrict__ sid)
{
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.total; g += gridDim.x * blockDim.x) {
        const uint32_t v = vals[g];
        sid[g] = v < bt.total ? segment_of(bt.off, bt.scenes, v) : 0u;  // (out of range only after a failed pass)
    }
}

// Each scene's sorted keys: position g of the final order lies in scene sc (the order
// is grouped by scene); its key is that of input element order[g].
template <typename K>
__global__ void __launch_bounds__(kBatchBlock) k_batch_keys(BatchTable bt, const K* __restrict__ keys_in,
                                                            const uint32_t* __restrict__ order)
{
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.total; g += gridDim.x * blockDim.x) {
        const uint32_t sc = segment_of(bt.off, bt.scenes, g);
        const uint32_t v = order[g];
        static_cast<K*>(bt.s[sc].keys)[g - bt.off[sc]] = v < bt.total ? keys_in[v] : (K)0;
    }
}

template <typename K>
__global__ void __launch_bounds__(256) k_batch_topology(BatchTable bt, int* __restrict__ counters,
                                                        const uint32_t* __restrict__ batch_status)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t inner_total = bt.total - bt.scenes;
    if (j >= inner_total) return;
    if (sort_timed_out(batch_status)) return;
    const uint32_t sc = segment_of(bt.inner_off, bt.scenes, j);
    const BatchScene& S = bt.s[sc];
    const int nn = (int)(bt.off[sc + 1] - bt.off[sc]);
    topology_node(static_cast<const K*>(S.keys), nn, (int)(j - bt.inner_off[sc]), S.children, S.parents_leaf,
                  S.parents_internal, counters + bt.inner_off[sc], reinterpret_cast<float4*>(S.nodes));
}

__global__ void __launch_bounds__(kBatchRefitBlock) k_batch_refit(BatchTable bt, const uint32_t* __restrict__ order,
                                                                  int* __restrict__ counters,
                                                                  const uint32_t* __restrict__ batch_status)
{
    __shared__ int s_count[kBatchRefitBlock];
    __shared__ float s_box[2 * kBatchRefitBlock][6];
    s_count[threadIdx.x] = 0;
    __syncthreads();
    if (sort_timed_out(batch_status)) return;  // (uniform: set before this launch)
    const uint32_t sc = segment_of(bt.block_off, bt.scenes, blockIdx.x);
    const BatchScene& S = bt.s[sc];
    const uint32_t n = bt.off[sc + 1] - bt.off[sc];
    const uint32_t base = (blockIdx.x - bt.block_off[sc]) * kBatchRefitBlock;
    const uint32_t i = base + threadIdx.x;
    if (i >= n) return;
    const uint32_t v = order[bt.off[sc] + i];
    const uint32_t src = v >= bt.off[sc] ? v - bt.off[sc] : n;  // n: out of range, reported by the walk
    gather_refit_leaf(S.tris_in, src, i, n, base, min(n, base + (uint32_t)kBatchRefitBlock), S.tris_out,
                          S.parents_leaf, S.parents_internal, counters + bt.inner_off[sc], S.nodes, S.node_boxes,
                          S.status, s_count, s_box);
}

__global__ void k_batch_status(BatchTable bt, const uint32_t* __restrict__ batch_status)
{
    const uint32_t w = *batch_status;
    for (uint32_t sc = threadIdx.x; sc < bt.scenes; sc += blockDim.x)
        if (w) atomicOr(bt.s[sc].status, w);
}

template <typename K>
struct BatchScratch {
    K* keys[3];  // [0]: keys in input order (kept), [1], [2]: the passes' ping-pong
    uint32_t* vals[2];
    uint32_t* sid[2];
    uint32_t* hist;
    uint32_t* offsets;
    uint32_t* zero;  // tile counters + look-back words, zeroed by k_batch_morton
    size_t zero_words;
    int* counters;
    uint32_t* status;  // the batch's own status word (sort and input errors)
    float* tris_copy;  // inputs of in-place scenes
};

template <typename K>
size_t batch_layout(uint64_t total, uint32_t scenes, void* base, BatchScratch<K>* out)
{
    constexpr int P = KeyTraits<K>::passes;
    Carver c(base);
    BatchScratch<K> s;
    const size_t tiles = (size_t)((total + kSortTile - 1) / kSortTile);
    for (int k = 0; k < 3; ++k) s.keys[k] = c.take<K>(total);
    s.vals[0] = c.take<uint32_t>(total);
    s.vals[1] = c.take<uint32_t>(total);
    s.sid[0] = c.take<uint32_t>(total);
    s.sid[1] = c.take<uint32_t>(total);
    s.hist = c.take<uint32_t>((size_t)(P + 1) * kRadix);
    s.offsets = c.take<uint32_t>((size_t)(P + 1) * kRadix);
    s.zero_words = 32 + (size_t)(P + 1) * tiles * kRadix;
    s.zero = c.take<uint32_t>(s.zero_words);
    s.counters = c.take<int>(total - scenes);
    s.status = c.take<uint32_t>(4);
    s.tris_copy = c.take<float>(10ull * total);
    if (out) *out = s;
    return c.used();
}

template <typename K>
int batch_impl(BatchTable& bt, const cpt_triangle* const* tris_in, cpt_bvh* const* bvhs, void* scratch,
               cudaStream_t stream)
{
    constexpr int P = KeyTraits<K>::passes;
    BatchScratch<K> s;
    batch_layout<K>(bt.total, bt.scenes, scratch, &s);
    // in-place scenes (input = the output's triangle array) gather from a copy
    for (uint32_t sc = 0; sc < bt.scenes; ++sc) {
        if (reinterpret_cast<const void*>(tris_in[sc]) != bvhs[sc]->tris) continue;
        float* dst = s.tris_copy + 10ull * bt.off[sc];
        CPT_CUDA_TRY(cudaMemcpyAsync(dst, tris_in[sc], sizeof(cpt_triangle) * (size_t)(bt.off[sc + 1] - bt.off[sc]),
                                     cudaMemcpyDeviceToDevice, stream));
        bt.s[sc].tris_in = dst;
    }
    // histograms and the batch status word are adjacent: one clear
    CPT_CUDA_TRY(cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * (P + 1) * kRadix, stream));
    CPT_CUDA_TRY(cudaMemsetAsync(s.status, 0, 4 * sizeof(uint32_t), stream));
    const int sms = sm_count();
    const int grid = (int)std::min<uint64_t>((bt.total + kBatchBlock - 1) / kBatchBlock, (uint64_t)sms * 8);
    {
        CPT_PROF(K_MORTON, stream);
        k_batch_morton<K><<<grid, kBatchBlock, 0, stream>>>(bt, s.keys[0], s.hist, s.zero, s.zero_words, s.status);
    }
    CPT_LAUNCH_CHECK();
    {
        CPT_PROF(K_SCAN, stream);
        k_scan_offsets<<<P + 1, kRadix, 0, stream>>>(s.hist, s.offsets);
    }
    CPT_LAUNCH_CHECK();
    const uint32_t tiles = (bt.total + kSortTile - 1) / kSortTile;
    uint32_t* lookback = s.zero + 32;
    if constexpr (sizeof(K) == 8) {
        // as 32-bit halves (in keys[1]); only the order is needed, k_batch_keys gathers
        // each scene's sorted keys from keys[0] afterwards
        if (const int rc = onesweep_sort64_halves(reinterpret_cast<const uint64_t*>(s.keys[0]),
                                                  reinterpret_cast<uint64_t*>(s.keys[1]), bt.total, bt.total, nullptr,
                                                  s.vals, s.offsets, lookback, s.zero, s.status, SortWait(), false,
                                                  true, stream))
            return rc;
    } else {
        const size_t smem = onesweep_smem<K>();
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // key passes: keys[0] -> keys[1] -> keys[2] -> keys[1] ...; values 0 -> 1 -> 0 ...
        for (int p = 0; p < P; ++p) {
            const K* kin = p == 0 ? s.keys[0] : s.keys[1 + ((p + 1) & 1)];
            K* kout = s.keys[1 + (p & 1)];
            const uint32_t* vin = p == 0 ? nullptr : s.vals[(p + 1) & 1];
            uint32_t* vout = s.vals[p & 1];
            uint32_t* lb = lookback + (size_t)p * tiles * kRadix;
            CPT_PROF(K_ONESWEEP, stream);
            if (p == 0)
                k_onesweep<K, true><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, bt.total, nullptr, 8 * p,
                                                                         s.offsets + p * kRadix, lb, s.zero + p,
                                                                         s.status);
            else
                k_onesweep<K, false><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, bt.total, nullptr,
                                                                          8 * p, s.offsets + p * kRadix, lb,
                                                                          s.zero + p, s.status);
            CPT_LAUNCH_CHECK();
        }
    }
    const uint32_t* order = s.vals[(P - 1) & 1];
    if (bt.scenes > 1) {  // the scene digit: one more stable pass
        k_batch_scene_ids<<<grid, kBatchBlock, 0, stream>>>(bt, order, s.sid[0]);
        CPT_LAUNCH_CHECK();
        const size_t smem32 = onesweep_smem<uint32_t>();
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<uint32_t, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem32));
        uint32_t* vout = s.vals[P & 1];
        {
            CPT_PROF(K_ONESWEEP, stream);
            k_onesweep<uint32_t, false><<<tiles, kSortBlock, smem32, stream>>>(
                s.sid[0], order, s.sid[1], vout, bt.total, nullptr, 0, s.offsets + P * kRadix,
                lookback + (size_t)P * tiles * kRadix, s.zero + P, s.status);
        }
        CPT_LAUNCH_CHECK();
        order = vout;
    }
    k_batch_keys<K><<<grid, kBatchBlock, 0, stream>>>(bt, s.keys[0], order);
    CPT_LAUNCH_CHECK();
    const uint32_t inner_total = bt.total - bt.scenes;
    {
        CPT_PROF(K_TOPOLOGY, stream);
        k_batch_topology<K><<<(inner_total + 255) / 256, 256, 0, stream>>>(bt, s.counters, s.status);
    }
    CPT_LAUNCH_CHECK();
    {
        CPT_PROF(K_GATHER_REFIT, stream);
        k_batch_refit<<<bt.block_off[bt.scenes], kBatchRefitBlock, 0, stream>>>(bt, order, s.counters, s.status);
    }
    CPT_LAUNCH_CHECK();
    k_batch_status<<<1, 64, 0, stream>>>(bt, s.status);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

// Host-side scene table and argument checks shared by the size query and the build.
int make_table(const uint32_t* n, uint32_t scenes, BatchTable& bt)
{
    if (!n || scenes == 0 || scenes > CPT_MAX_BATCH_SCENES) return CPT_ERR_INVALID_ARGUMENT;
    uint64_t total = 0, blocks = 0;
    bt.scenes = scenes;
    for (uint32_t sc = 0; sc < scenes; ++sc) {
        if (n[sc] < 2 || n[sc] > kMaxTriangles) return CPT_ERR_INVALID_ARGUMENT;
        bt.off[sc] = (uint32_t)total;
        bt.inner_off[sc] = (uint32_t)(total - sc);
        bt.block_off[sc] = (uint32_t)blocks;
        total += n[sc];
        blocks += (n[sc] + kBatchRefitBlock - 1) / kBatchRefitBlock;
        if (total > kMaxTriangles) return CPT_ERR_INVALID_ARGUMENT;  // 30-bit counts in the look-back words
    }
    bt.off[scenes] = (uint32_t)total;
    bt.inner_off[scenes] = (uint32_t)(total - scenes);
    bt.block_off[scenes] = (uint32_t)blocks;
    bt.total = (uint32_t)total;
    return CPT_OK;
}

}  // namespace
}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_lbvh_batch_scratch_bytes(const uint32_t* n, uint32_t scenes, int morton_bits)
{
    if (morton_bits != 30 && morton_bits != 63) return 0;
    BatchTable bt;
    if (make_table(n, scenes, bt) != CPT_OK) return 0;
    return morton_bits == 30 ? batch_layout<uint32_t>(bt.total, scenes, nullptr, nullptr)
                             : batch_layout<uint64_t>(bt.total, scenes, nullptr, nullptr);
}

extern "C" int cpt_lbvh_build_batch(const cpt_triangle* const* tris_in, const uint32_t* n, uint32_t scenes,
                                    const float* boxes, int morton_bits, cpt_bvh* const* bvhs, void* scratch,
                                    size_t scratch_bytes, uint32_t flags, cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_build_batch");
    if (!tris_in || !boxes || !bvhs || !scratch || (morton_bits != 30 && morton_bits != 63))
        return CPT_ERR_INVALID_ARGUMENT;
    if (flags & ~CPT_BUILD_CHECK) return CPT_ERR_INVALID_ARGUMENT;
    static BatchTable bt;  // ~7 KB: filled on the host, passed by value to the kernels
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    int rc = make_table(n, scenes, bt);
    if (rc != CPT_OK) return rc;
    if (reinterpret_cast<uintptr_t>(scratch) & 255) return CPT_ERR_INVALID_ARGUMENT;
    const size_t need = cpt_lbvh_batch_scratch_bytes(n, scenes, morton_bits);
    if (scratch_bytes < need) return CPT_ERR_SCRATCH_TOO_SMALL;
    for (uint32_t sc = 0; sc < scenes; ++sc) {
        cpt_bvh* b = bvhs[sc];
        if (!b || !tris_in[sc]) return CPT_ERR_INVALID_ARGUMENT;
        if (b->n != n[sc] || b->morton_bits != morton_bits || !b->tris || !b->keys || !b->children ||
            !b->parents_leaf || !b->parents_internal || !b->node_boxes || !b->nodes || !b->status)
            return CPT_ERR_INVALID_ARGUMENT;
        if ((reinterpret_cast<uintptr_t>(tris_in[sc]) & 15) || (reinterpret_cast<uintptr_t>(b->nodes) & 15) ||
            (reinterpret_cast<uintptr_t>(b->tris) & 15))
            return CPT_ERR_INVALID_ARGUMENT;
    }
    for (uint32_t sc = 0; sc < scenes; ++sc) {
        cpt_bvh* b = bvhs[sc];
        b->split_nodes = nullptr;  // split and wide trees of the previous build are stale
        b->split_capacity = 0;
        b->wide_nodes = nullptr;
        b->wide_tris = nullptr;
        b->wide_capacity = 0;
        BatchScene& S = bt.s[sc];
        S.tris_in = reinterpret_cast<const float*>(tris_in[sc]);
        S.tris_out = reinterpret_cast<float*>(b->tris);
        S.keys = b->keys;
        S.children = b->children;
        S.parents_leaf = b->parents_leaf;
        S.parents_internal = b->parents_internal;
        S.node_boxes = b->node_boxes;
        S.nodes = static_cast<float*>(b->nodes);
        S.status = b->status;
        const float* bx = boxes + 6 * (size_t)sc;
        for (int a = 0; a < 3; ++a) {  // as the single build's host box (lbvh.cu build_impl)
            S.mn[a] = bx[a];
            S.inv[a] = 1.0f / (bx[3 + a] - bx[a]);
        }
    }
    rc = morton_bits == 30 ? batch_impl<uint32_t>(bt, tris_in, bvhs, scratch, stream)
                           : batch_impl<uint64_t>(bt, tris_in, bvhs, scratch, stream);
    if (rc != CPT_OK || !(flags & CPT_BUILD_CHECK)) return rc;
    // per scene: device status, then the root-volume self-check of BVHBuilder.cu:258-265
    for (uint32_t sc = 0; sc < scenes; ++sc) {
        rc = cpt_status_check(bvhs[sc]->status, stream);
        if (rc != CPT_OK) return rc;
        cpt_bbox root;
        CPT_CUDA_TRY(cudaMemcpyAsync(&root, bvhs[sc]->node_boxes, sizeof(root), cudaMemcpyDeviceToHost, stream));
        CPT_CUDA_TRY(cudaStreamSynchronize(stream));
        const float* eb = boxes + 6 * (size_t)sc;
        const float ve = (eb[3] - eb[0]) * (eb[4] - eb[1]) * (eb[5] - eb[2]);
        const float vr = (root.max[0] - root.min[0]) * (root.max[1] - root.min[1]) * (root.max[2] - root.min[2]);
        if (!(fabsf(ve - vr) <= 1e-7f)) return CPT_ERR_CHECK_FAILED;
    }
    return CPT_OK;
}
