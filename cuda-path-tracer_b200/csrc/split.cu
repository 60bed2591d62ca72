// Split traversal BVH (cpt_lbvh_split): a second, traversal-only LBVH over pieces
// of the triangles, for scenes whose long thin triangles (the hairball) have
// boxes far larger than the triangles: every ray crossing such a box must test
// the triangle. Cutting a long triangle into pieces along its longest axis and
// giving each piece the box of the triangle clipped to its slab shrinks the boxes
// a ray crosses roughly by the piece count.
//
// The reference-format BVH (cpt_lbvh_build) is untouched and stays bit-exact;
// this one is built from its Morton-sorted triangles and only changes which
// nodes a ray visits. Its leaves hold the whole triangle (v0, the triangle's
// sorted index, v1 - v0, v2 - v0), so a ray tests the same triangle with the same
// arithmetic and reports the same index; the closest hit is the same triangle
// unless two triangles are hit at exactly the same distance, where the visiting
// order decides. Piece boxes contain the exact clipped triangle: along the split
// axis they are the slab bounds, across it the clipped polygon's extent widened
// by 2^-20 of the coordinates' magnitude (and kept inside the triangle's box), so
// rounding in the clipping cannot drop a hit.
//
// Steps (all on the device, one stream, the piece count never leaves the GPU):
//   k_split_weight/total  w_i = sqrt(max(0, area(box_i) - 2 area(tri_i))), sum in fixed order
//   k_split_count         pieces s_i = 1 + min(63, floor(extra * w_i / sum w)) -> sum s_i <= n + extra
//   k_split_scan_tiles    piece offsets of each 4096-triangle tile, total piece count
//   k_split_emit          pieces: clipped boxes, Morton keys of their centres in the root box,
//                         digit histograms, zeroed look-back state
//   k_scan_offsets, k_onesweep x P, k_topology   as the main build, on the device count
//   k_split_refit         leaf slots + bottom-up boxes into the 96-B traversal nodes
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"
#include "lbvh_common.cuh"
#include "onesweep.cuh"

namespace cpt {
namespace {

constexpr int kSplitBlock = 256;
constexpr int kMaxPieces = 64;
constexpr int kScanItems = 16;
constexpr int kScanTile = kSplitBlock * kScanItems;  // triangles per emit / count tile
constexpr int kWeightBlocks = 1024;

__device__ __forceinline__ void tri_box(const cpt_triangle& t, float lo[3], float hi[3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lo[a] = fminf(fminf(t.v0[a], t.v1[a]), t.v2[a]);
        hi[a] = fmaxf(fmaxf(t.v0[a], t.v1[a]), t.v2[a]);
    }
}

__device__ __forceinline__ float split_weight(const cpt_triangle& t)
{
    float lo[3], hi[3];
    tri_box(t, lo, hi);
    const float ex = hi[0] - lo[0], ey = hi[1] - lo[1], ez = hi[2] - lo[2];
    const float box_area = 2.0f * (ex * ey + ey * ez + ez * ex);
    float e1[3], e2[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) { e1[a] = t.v1[a] - t.v0[a]; e2[a] = t.v2[a] - t.v0[a]; }
    const float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2];
    const float cz = e1[0] * e2[1] - e1[1] * e2[0];
    const float tri_area = 0.5f * sqrtf(cx * cx + cy * cy + cz * cz);
    const float w = sqrtf(fmaxf(box_area - 2.0f * tri_area, 0.0f));
    return isfinite(w) ? w : 0.0f;
}

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double s_warp[kSplitBlock / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kSplitBlock / 32; ++k) t += s_warp[k];
    return t;  // valid on thread 0
}

__global__ void __launch_bounds__(kSplitBlock) k_split_weight(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                              double* __restrict__ partial)
{
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * kSplitBlock + threadIdx.x; i < n; i += gridDim.x * kSplitBlock)
        acc += (double)split_weight(tris[i]);
    const double t = block_sum(acc);
    if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

__global__ void k_split_total(const double* __restrict__ partial, int blocks, double* __restrict__ total)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += partial[b];
    *total = t;
}

// Exclusive scan of one value per thread over the block; returns the block total
// through *total (all threads).
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t s_warp[kSplitBlock / 32 + 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int k = 0; k < kSplitBlock / 32; ++k) {
            const uint32_t t = s_warp[k];
            s_warp[k] = run;
            run += t;
        }
        s_warp[kSplitBlock / 32] = run;
    }
    __syncthreads();
    const uint32_t r = s_warp[warp] + x - v;
    *total = s_warp[kSplitBlock / 32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ uint32_t piece_count(const cpt_triangle& t, double total, double extra)
{
    if (!(total > 0.0)) return 1u;
    const double share = extra * (double)split_weight(t) / total;
    const double extra_i = floor(share);
    return 1u + (uint32_t)fmin(extra_i, (double)(kMaxPieces - 1));
}

__global__ void __launch_bounds__(kSplitBlock) k_split_count(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                             const double* __restrict__ total, double extra,
                                                             uint32_t* __restrict__ counts,
                                                             uint32_t* __restrict__ tile_sums)
{
    const double tot = *total;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t sum = 0;
#pragma unroll 4
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        if (i >= n) break;
        const uint32_t c = piece_count(tris[i], tot, extra);
        counts[i] = c;
        sum += c;
    }
    uint32_t block_total;
    block_exclusive_scan(sum, &block_total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = block_total;
}

// Tile sums -> exclusive tile offsets (in place) and the piece count; one block.
__global__ void __launch_bounds__(1024) k_split_scan_tiles(uint32_t* __restrict__ tile_sums, uint32_t tiles,
                                                           uint32_t capacity, uint32_t* __restrict__ n_pieces,
                                                           uint32_t* __restrict__ status)
{
    __shared__ uint32_t s_part[1024];
    const int per = (int)((tiles + 1023) / 1024);
    uint32_t loc = 0;
    for (int k = 0; k < per; ++k) {
        const uint32_t t = threadIdx.x * per + k;
        if (t < tiles) loc += tile_sums[t];
    }
    s_part[threadIdx.x] = loc;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int k = 0; k < 1024; ++k) {
            const uint32_t v = s_part[k];
            s_part[k] = run;
            run += v;
        }
        if (run > capacity) {  // cannot happen (the shares sum to at most `extra`); stay in bounds
            atomicOr(status, CPT_STATUS_BAD_INDEX);
            run = capacity;
        }
        *n_pieces = run;
    }
    __syncthreads();
    uint32_t run = s_part[threadIdx.x];
    for (int k = 0; k < per; ++k) {
        const uint32_t t = threadIdx.x * per + k;
        if (t < tiles) {
            const uint32_t v = tile_sums[t];
            tile_sums[t] = run;
            run += v;
        }
    }
}

// Box of triangle t clipped to lo_s <= x_axis <= hi_s (conservative, see the file comment).
__device__ __forceinline__ void clip_box(const cpt_triangle& t, int axis, float lo_s, float hi_s, const float tlo[3],
                                         const float thi[3], float bmn[3], float bmx[3])
{
    float poly[5][3], tmp[5][3];
    int np = 3;
#pragma unroll
    for (int a = 0; a < 3; ++a) { poly[0][a] = t.v0[a]; poly[1][a] = t.v1[a]; poly[2][a] = t.v2[a]; }
    // clip against x >= lo_s, then x <= hi_s (Sutherland-Hodgman)
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const float plane = side == 0 ? lo_s : hi_s;
        int nt = 0;
        for (int k = 0; k < np; ++k) {
            const float* a = poly[k];
            const float* b = poly[(k + 1) % np];
            const float da = side == 0 ? a[axis] - plane : plane - a[axis];
            const float db = side == 0 ? b[axis] - plane : plane - b[axis];
            const bool ina = da >= 0.f, inb = db >= 0.f;
            if (ina && nt < 5) {
                tmp[nt][0] = a[0]; tmp[nt][1] = a[1]; tmp[nt][2] = a[2];
                ++nt;
            }
            if (ina != inb && nt < 5) {
                const float s = da / (da - db);
#pragma unroll
                for (int c = 0; c < 3; ++c) tmp[nt][c] = a[c] + s * (b[c] - a[c]);
                ++nt;
            }
        }
        np = nt;
        for (int k = 0; k < np; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) poly[k][c] = tmp[k][c];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) { bmn[a] = tlo[a]; bmx[a] = thi[a]; }
    if (np > 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float mn = poly[0][a], mx = poly[0][a];
            for (int k = 1; k < np; ++k) { mn = fminf(mn, poly[k][a]); mx = fmaxf(mx, poly[k][a]); }
            const float eps = (fabsf(mn) + fabsf(mx) + (thi[a] - tlo[a])) * 9.5367431640625e-07f;  // 2^-20
            bmn[a] = fmaxf(mn - eps, tlo[a]);
            bmx[a] = fminf(mx + eps, thi[a]);
        }
    }
    bmn[axis] = fmaxf(lo_s, tlo[axis]);
    bmx[axis] = fminf(hi_s, thi[axis]);
}

template <typename K>
__global__ void __launch_bounds__(kSplitBlock) k_split_emit(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                            const uint32_t* __restrict__ counts,
                                                            const uint32_t* __restrict__ tile_offsets,
                                                            const cpt_bbox* __restrict__ root, uint32_t capacity,
                                                            float4* __restrict__ pieces, K* __restrict__ keys,
                                                            uint32_t* __restrict__ hist, uint32_t* __restrict__ zero,
                                                            size_t zero_words, uint32_t* __restrict__ status)
{
    constexpr int P = KeyTraits<K>::passes;
    constexpr int order = KeyTraits<K>::order;
    __shared__ uint32_t s_hist[P * kRadix];
    for (int i = threadIdx.x; i < P * kRadix; i += kSplitBlock) s_hist[i] = 0;
    {
        const size_t gtid = (size_t)blockIdx.x * kSplitBlock + threadIdx.x, gsize = (size_t)gridDim.x * kSplitBlock;
        for (size_t i = gtid; i < zero_words; i += gsize) zero[i] = 0;
    }
    float rmn[3], rinv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        rmn[a] = root->min[a];
        rinv[a] = __frcp_rn(__fsub_rn(root->max[a], root->min[a]));
    }
    const uint32_t cells = 1u << order;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t sum = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) sum += counts[i];
    }
    uint32_t block_total;
    uint32_t off = tile_offsets[blockIdx.x] + block_exclusive_scan(sum, &block_total);
    bool overflow = false;
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        if (i >= n) break;
        const cpt_triangle t = tris[i];
        const uint32_t s = counts[i];
        float tlo[3], thi[3];
        tri_box(t, tlo, thi);
        int axis = 0;
        float ext = thi[0] - tlo[0];
        if (thi[1] - tlo[1] > ext) { axis = 1; ext = thi[1] - tlo[1]; }
        if (thi[2] - tlo[2] > ext) { axis = 2; ext = thi[2] - tlo[2]; }
        for (uint32_t p = 0; p < s; ++p, ++off) {
            if (off >= capacity) { overflow = true; break; }
            float bmn[3], bmx[3];
            if (s == 1) {
#pragma unroll
                for (int a = 0; a < 3; ++a) { bmn[a] = tlo[a]; bmx[a] = thi[a]; }
            } else {
                const float lo_s = p == 0 ? tlo[axis] : tlo[axis] + ext * ((float)p / (float)s);
                const float hi_s = p + 1 == s ? thi[axis] : tlo[axis] + ext * ((float)(p + 1) / (float)s);
                clip_box(t, axis, lo_s, hi_s, tlo, thi, bmn, bmx);
            }
            pieces[2 * (size_t)off] = make_float4(bmn[0], bmn[1], bmn[2], __uint_as_float(i));
            pieces[2 * (size_t)off + 1] = make_float4(bmx[0], bmx[1], bmx[2], 0.f);
            uint32_t q[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float c = 0.5f * (bmn[a] + bmx[a]);
                q[a] = quantize(__fmul_rn(__fsub_rn(c, rmn[a]), rinv[a]), cells);
            }
            const uint64_t key = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
            keys[off] = (K)key;
#pragma unroll
            for (int pp = 0; pp < P; ++pp) atomicAdd(&s_hist[pp * kRadix + (uint32_t)((key >> (8 * pp)) & 0xFF)], 1u);
        }
    }
    if (overflow) atomicOr(status, CPT_STATUS_BAD_INDEX);
    __syncthreads();
    for (int i = threadIdx.x; i < P * kRadix; i += kSplitBlock)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

__device__ __forceinline__ Box piece_box(const float4* pieces, uint32_t r, bool coherent)
{
    const float4 a = coherent ? __ldcg(pieces + 2 * (size_t)r) : pieces[2 * (size_t)r];
    const float4 b = coherent ? __ldcg(pieces + 2 * (size_t)r + 1) : pieces[2 * (size_t)r + 1];
    Box x;
    x.mn[0] = a.x; x.mn[1] = a.y; x.mn[2] = a.z;
    x.mx[0] = b.x; x.mx[1] = b.y; x.mx[2] = b.z;
    return x;
}

// Leaf i (sorted piece order[i]): its slot is the whole triangle, its box the
// piece's; then the bottom-up walk of k_gather_refit with the sibling leaf's box
// read from the leaf box array.
__global__ void __launch_bounds__(256) k_split_refit(const cpt_triangle* __restrict__ tris, const float4* __restrict__ pieces,
                                                     const uint32_t* __restrict__ order,
                                                     const uint32_t* __restrict__ n_pieces,
                                                     const uint32_t* __restrict__ children,
                                                     const uint32_t* __restrict__ parents_leaf,
                                                     const uint32_t* __restrict__ parents_internal,
                                                     int* __restrict__ counters, float* __restrict__ nodes,
                                                     cpt_bbox* __restrict__ node_boxes, float4* __restrict__ leaf_boxes,
                                                     uint32_t n_tris, uint32_t* __restrict__ status)
{
    const uint32_t n = *n_pieces;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || n < 2) return;
    uint32_t src = order[i];
    if (src >= n) {
        atomicOr(status, CPT_STATUS_BAD_INDEX);
        src = n - 1;
    }
    Box box = piece_box(pieces, src, false);
    uint32_t tri = __float_as_uint(pieces[2 * (size_t)src].w);
    if (tri >= n_tris) {
        atomicOr(status, CPT_STATUS_BAD_INDEX);
        tri = n_tris - 1;
    }
    leaf_boxes[2 * (size_t)i] = make_float4(box.mn[0], box.mn[1], box.mn[2], 0.f);
    leaf_boxes[2 * (size_t)i + 1] = make_float4(box.mx[0], box.mx[1], box.mx[2], 0.f);
    const cpt_triangle t = tris[tri];
    float slot[10] = {t.v0[0], t.v0[1], t.v0[2], __uint_as_float(tri),
                      __fsub_rn(t.v1[0], t.v0[0]), __fsub_rn(t.v1[1], t.v0[1]), __fsub_rn(t.v1[2], t.v0[2]),
                      __fsub_rn(t.v2[0], t.v0[0]), __fsub_rn(t.v2[1], t.v0[1]), __fsub_rn(t.v2[2], t.v0[2])};
    __threadfence();
    uint32_t child = i;
    uint32_t p = parents_leaf[i];
    while (p != CPT_INVALID_INDEX) {
        if (p >= n - 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }
        const uint32_t word = children[p];
        const uint32_t left = word >> 2;
        const int side = left == child ? 0 : 1;
        float* node = nodes + 24 * (size_t)p;
        store_slot(node, side, slot);
        __threadfence();
        const int arrived = atomicAdd(&counters[p], 1);
        if (arrived == 0) return;
        if (arrived != 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }
        __threadfence();
        const uint32_t sib = left + (uint32_t)(1 - side);
        const bool sib_internal = (word >> (1 - side)) & 1u;
        Box sb;
        if (sib_internal) {
            const float2* q = reinterpret_cast<const float2*>(node_boxes + sib);
            const float2 x0 = __ldcg(q), x1 = __ldcg(q + 1), x2 = __ldcg(q + 2);
            sb.mn[0] = x0.x; sb.mn[1] = x0.y; sb.mn[2] = x1.x; sb.mx[0] = x1.y; sb.mx[1] = x2.x; sb.mx[2] = x2.y;
        } else {
            sb = piece_box(leaf_boxes, sib, true);
        }
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            box.mn[ax] = fminf(box.mn[ax], sb.mn[ax]);
            box.mx[ax] = fmaxf(box.mx[ax], sb.mx[ax]);
        }
        float2* ob = reinterpret_cast<float2*>(node_boxes + p);
        ob[0] = make_float2(box.mn[0], box.mn[1]);
        ob[1] = make_float2(box.mn[2], box.mx[0]);
        ob[2] = make_float2(box.mx[1], box.mx[2]);
#pragma unroll
        for (int k = 0; k < 3; ++k) { slot[k] = box.mn[k]; slot[3 + k] = box.mx[k]; }
        slot[6] = slot[7] = slot[8] = slot[9] = 0.0f;
        child = p;
        p = parents_internal[p];
    }
}

template <typename K>
struct SplitScratch {
    double* partial;
    double* total;
    uint32_t* counts;
    uint32_t* tile_sums;
    uint32_t* n_pieces;
    float4* pieces;
    K* keys[2];
    uint32_t* vals[2];
    uint32_t* hist;
    uint32_t* offsets;
    uint32_t* zero;
    size_t zero_words;
    uint32_t* children;
    uint32_t* parents_leaf;
    uint32_t* parents_internal;
    int* counters;
    cpt_bbox* node_boxes;
    float4* leaf_boxes;
};

template <typename K>
size_t split_layout(uint32_t n, uint32_t cap, void* base, SplitScratch<K>* out)
{
    constexpr int P = KeyTraits<K>::passes;
    Carver c(base);
    SplitScratch<K> s;
    const uint32_t ctiles = (n + kScanTile - 1) / kScanTile;
    const size_t sort_tiles = (cap + kSortTile - 1) / kSortTile;
    s.partial = c.take<double>(kWeightBlocks);
    s.total = c.take<double>(1);
    s.counts = c.take<uint32_t>(n);
    s.tile_sums = c.take<uint32_t>(ctiles);
    s.n_pieces = c.take<uint32_t>(1);
    s.pieces = c.take<float4>(2ull * cap);
    s.keys[0] = c.take<K>(cap);
    s.keys[1] = c.take<K>(cap);
    s.vals[0] = c.take<uint32_t>(cap);
    s.vals[1] = c.take<uint32_t>(cap);
    s.hist = c.take<uint32_t>((size_t)P * kRadix);
    s.offsets = c.take<uint32_t>((size_t)P * kRadix);
    s.zero_words = 32 + (size_t)P * sort_tiles * kRadix;
    s.zero = c.take<uint32_t>(s.zero_words);
    s.children = c.take<uint32_t>(cap);
    s.parents_leaf = c.take<uint32_t>(cap);
    s.parents_internal = c.take<uint32_t>(cap);
    s.counters = c.take<int>(cap);
    s.node_boxes = c.take<cpt_bbox>(cap);
    s.leaf_boxes = c.take<float4>(2ull * cap);
    if (out) *out = s;
    return c.used();
}

inline uint64_t split_capacity(uint32_t n, float extra_ratio)
{
    const double r = extra_ratio > 0.f ? (double)extra_ratio : 0.0;
    return (uint64_t)n + (uint64_t)floor(r * (double)n);
}

template <typename K>
int split_impl(cpt_bvh* bvh, uint32_t cap, void* nodes, void* scratch, cudaStream_t stream)
{
    constexpr int P = KeyTraits<K>::passes;
    const uint32_t n = bvh->n;
    SplitScratch<K> s;
    split_layout<K>(n, cap, scratch, &s);
    const uint32_t ctiles = (n + kScanTile - 1) / kScanTile;
    const double extra = (double)(cap - n);
    CPT_CUDA_TRY(cudaMemsetAsync(s.hist, 0, sizeof(uint32_t) * P * kRadix, stream));
    k_split_weight<<<kWeightBlocks, kSplitBlock, 0, stream>>>(bvh->tris, n, s.partial);
    CPT_LAUNCH_CHECK();
    k_split_total<<<1, 32, 0, stream>>>(s.partial, kWeightBlocks, s.total);
    CPT_LAUNCH_CHECK();
    k_split_count<<<ctiles, kSplitBlock, 0, stream>>>(bvh->tris, n, s.total, extra, s.counts, s.tile_sums);
    CPT_LAUNCH_CHECK();
    k_split_scan_tiles<<<1, 1024, 0, stream>>>(s.tile_sums, ctiles, cap, s.n_pieces, bvh->status);
    CPT_LAUNCH_CHECK();
    k_split_emit<K><<<ctiles, kSplitBlock, 0, stream>>>(bvh->tris, n, s.counts, s.tile_sums, bvh->node_boxes, cap,
                                                        s.pieces, s.keys[0], s.hist, s.zero, s.zero_words,
                                                        bvh->status);
    CPT_LAUNCH_CHECK();
    k_scan_offsets<<<P, kRadix, 0, stream>>>(s.hist, s.offsets);
    CPT_LAUNCH_CHECK();
    const size_t smem = onesweep_smem<K>();
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const uint32_t tiles = (cap + kSortTile - 1) / kSortTile;
    uint32_t* lookback = s.zero + 32;
    for (int p = 0; p < P; ++p) {
        const K* kin = s.keys[p & 1];
        K* kout = s.keys[(p + 1) & 1];
        const uint32_t* vin = p == 0 ? nullptr : s.vals[(p + 1) & 1];
        uint32_t* vout = s.vals[p & 1];
        uint32_t* lb = lookback + (size_t)p * tiles * kRadix;
        if (p == 0)
            k_onesweep<K, true><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, 0, s.n_pieces, 8 * p,
                                                                     s.offsets + p * kRadix, lb, s.zero + p,
                                                                     bvh->status);
        else
            k_onesweep<K, false><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, 0, s.n_pieces, 8 * p,
                                                                      s.offsets + p * kRadix, lb, s.zero + p,
                                                                      bvh->status);
        CPT_LAUNCH_CHECK();
    }
    const uint32_t* order = s.vals[(P - 1) & 1];
    const K* keys = s.keys[P & 1];
    k_topology<K><<<(cap + 255) / 256, 256, 0, stream>>>(keys, 0, s.n_pieces, s.children, s.parents_leaf,
                                                          s.parents_internal, s.counters, static_cast<float4*>(nodes));
    CPT_LAUNCH_CHECK();
    k_split_refit<<<(cap + 255) / 256, 256, 0, stream>>>(bvh->tris, s.pieces, order, s.n_pieces, s.children,
                                                          s.parents_leaf, s.parents_internal, s.counters,
                                                          static_cast<float*>(nodes), s.node_boxes, s.leaf_boxes, n,
                                                          bvh->status);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

}  // namespace
}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_lbvh_split_bytes(uint32_t n, int morton_bits, float extra_ratio, size_t* node_bytes)
{
    if (n < 2 || (morton_bits != 30 && morton_bits != 63)) return 0;
    const uint64_t cap = split_capacity(n, extra_ratio);
    if (cap >= (1ull << 31)) return 0;
    if (node_bytes) *node_bytes = align_up((size_t)(cap - 1) * 96, 256);
    return morton_bits == 30 ? split_layout<uint32_t>(n, (uint32_t)cap, nullptr, nullptr)
                             : split_layout<uint64_t>(n, (uint32_t)cap, nullptr, nullptr);
}

extern "C" int cpt_lbvh_split(cpt_bvh* bvh, float extra_ratio, void* nodes, size_t node_bytes, void* scratch,
                              size_t scratch_bytes, cudaStream_t stream)
{
    if (!bvh || !bvh->tris || !bvh->node_boxes || !bvh->status || !nodes || !scratch) return CPT_ERR_INVALID_ARGUMENT;
    if (!(extra_ratio >= 0.f) || !(extra_ratio <= 64.f)) return CPT_ERR_INVALID_ARGUMENT;
    size_t nb = 0;
    const size_t need = cpt_lbvh_split_bytes(bvh->n, bvh->morton_bits, extra_ratio, &nb);
    if (!need) return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < need || node_bytes < nb) return CPT_ERR_SCRATCH_TOO_SMALL;
    if ((reinterpret_cast<uintptr_t>(nodes) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 255))
        return CPT_ERR_INVALID_ARGUMENT;
    const uint32_t cap = (uint32_t)split_capacity(bvh->n, extra_ratio);
    const int rc = bvh->morton_bits == 30 ? split_impl<uint32_t>(bvh, cap, nodes, scratch, stream)
                                          : split_impl<uint64_t>(bvh, cap, nodes, scratch, stream);
    if (rc) return rc;
    bvh->split_nodes = nodes;
    bvh->split_capacity = cap;
    return CPT_OK;
}
