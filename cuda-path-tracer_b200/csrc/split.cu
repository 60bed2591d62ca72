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
//   k_split_first         each triangle's first piece (exclusive offsets, in place of the counts)
//   k_split_emit          pieces, 64 per thread (balanced however the triangles are cut):
//                         clipped boxes, Morton keys of their centres in the root box,
//                         digit histograms, zeroed look-back state
//   k_scan_offsets, k_onesweep x P, k_topology   as the main build, on the device count
//   k_split_refit         leaf slots + bottom-up boxes into the 96-B traversal nodes
//   k_treelet             (CPT_SPLIT_TREELET) treelet restructuring of the Karras topology
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

// Piece counts -> exclusive per-triangle piece offsets, in place (tile offsets from
// k_split_scan_tiles, a block scan inside the tile).
__global__ void __launch_bounds__(kSplitBlock) k_split_first(uint32_t n, uint32_t* __restrict__ counts,
                                                             const uint32_t* __restrict__ tile_offsets)
{
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t c[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        c[k] = i < n ? counts[i] : 0u;
        sum += c[k];
    }
    uint32_t block_total;
    uint32_t off = tile_offsets[blockIdx.x] + block_exclusive_scan(sum, &block_total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const uint32_t i = base + k;
        if (i < n) counts[i] = off;
        off += c[k];
    }
}

// Pieces of the triangles, kEmitPieces consecutive pieces per thread whatever the
// triangles they come from (a long hairball triangle is cut into up to 64 pieces):
// piece j belongs to the triangle i with first[i] <= j < first[i + 1], found once per
// thread by binary search. Writes the piece box, its Morton key and all the digit
// histograms of the sort, and zeroes the sort's look-back state.
constexpr int kEmitPieces = 64;

template <typename K>
__global__ void __launch_bounds__(kSplitBlock) k_split_emit(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                            const uint32_t* __restrict__ first,
                                                            const uint32_t* __restrict__ n_pieces,
                                                            const cpt_bbox* __restrict__ root,
                                                            float4* __restrict__ pieces, K* __restrict__ keys,
                                                            uint32_t* __restrict__ hist, uint32_t* __restrict__ zero,
                                                            size_t zero_words)
{
    constexpr int P = KeyTraits<K>::passes;
    constexpr int order = KeyTraits<K>::order;
    __shared__ uint32_t s_hist[P * kRadix];
    for (int i = threadIdx.x; i < P * kRadix; i += kSplitBlock) s_hist[i] = 0;
    {
        const size_t gtid = (size_t)blockIdx.x * kSplitBlock + threadIdx.x, gsize = (size_t)gridDim.x * kSplitBlock;
        for (size_t i = gtid; i < zero_words; i += gsize) zero[i] = 0;
    }
    __syncthreads();
    float rmn[3], rinv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        rmn[a] = root->min[a];
        rinv[a] = __frcp_rn(__fsub_rn(root->max[a], root->min[a]));
    }
    const uint32_t cells = 1u << order;
    const uint32_t np = *n_pieces;
    const uint64_t j0 = ((uint64_t)blockIdx.x * kSplitBlock + threadIdx.x) * kEmitPieces;
    if (j0 < np) {
        uint32_t lo = 0, hi = n - 1;  // the last triangle whose first piece is at or before j0
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (first[mid] <= j0) lo = mid;
            else hi = mid - 1;
        }
        uint32_t i = lo;
        uint32_t fi = first[i];
        uint32_t ei = i + 1 < n ? first[i + 1] : np;
        cpt_triangle t = tris[i];
        float tlo[3], thi[3];
        int axis = 0;
        float ext = 0.f;
        auto setup = [&]() {
            tri_box(t, tlo, thi);
            axis = 0;
            ext = thi[0] - tlo[0];
            if (thi[1] - tlo[1] > ext) { axis = 1; ext = thi[1] - tlo[1]; }
            if (thi[2] - tlo[2] > ext) { axis = 2; ext = thi[2] - tlo[2]; }
        };
        setup();
        const uint32_t jend = j0 + kEmitPieces < (uint64_t)np ? (uint32_t)(j0 + kEmitPieces) : np;
        for (uint32_t j = (uint32_t)j0; j < jend; ++j) {
            while (j >= ei && i + 1 < n) {  // the next triangle with pieces
                ++i;
                fi = ei;
                ei = i + 1 < n ? first[i + 1] : np;
                t = tris[i];
                setup();
            }
            const uint32_t s = ei - fi, p = j - fi;
            float bmn[3], bmx[3];
            if (s == 1) {
#pragma unroll
                for (int a = 0; a < 3; ++a) { bmn[a] = tlo[a]; bmx[a] = thi[a]; }
            } else {
                const float lo_s = p == 0 ? tlo[axis] : tlo[axis] + ext * ((float)p / (float)s);
                const float hi_s = p + 1 == s ? thi[axis] : tlo[axis] + ext * ((float)(p + 1) / (float)s);
                clip_box(t, axis, lo_s, hi_s, tlo, thi, bmn, bmx);
            }
            pieces[2 * (size_t)j] = make_float4(bmn[0], bmn[1], bmn[2], __uint_as_float(i));
            pieces[2 * (size_t)j + 1] = make_float4(bmx[0], bmx[1], bmx[2], 0.f);
            uint32_t q[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float c = 0.5f * (bmn[a] + bmx[a]);
                q[a] = quantize(__fmul_rn(__fsub_rn(c, rmn[a]), rinv[a]), cells);
            }
            const uint64_t key = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
            keys[j] = (K)key;
#pragma unroll
            for (int pp = 0; pp < P; ++pp) atomicAdd(&s_hist[pp * kRadix + (uint32_t)((key >> (8 * pp)) & 0xFF)], 1u);
        }
    }
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
// Leaves per block of k_split_refit: nodes whose leaf range (word 22 of the record,
// written by k_topology) lies inside the block complete in shared memory, as in the
// LBVH refit; the rest through the global acquire-release counters.
constexpr int kSplitRefitBlock = 64;

__global__ void __launch_bounds__(kSplitRefitBlock) k_split_refit(const cpt_triangle* __restrict__ tris, const float4* __restrict__ pieces,
                                                     const uint32_t* __restrict__ order,
                                                     const uint32_t* __restrict__ n_pieces,
                                                     const uint32_t* __restrict__ children,
                                                     const uint32_t* __restrict__ parents_leaf,
                                                     const uint32_t* __restrict__ parents_internal,
                                                     int* __restrict__ counters, float* __restrict__ nodes,
                                                     cpt_bbox* __restrict__ node_boxes, float4* __restrict__ leaf_boxes,
                                                     uint32_t n_tris, uint32_t* __restrict__ status)
{
    __shared__ int s_count[kSplitRefitBlock];
    __shared__ float s_box[2 * kSplitRefitBlock][6];  // [2 * (p - base) + side]: the first arriver's box
    const uint32_t base = blockIdx.x * kSplitRefitBlock;
    s_count[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t n = *n_pieces;
    const uint32_t i = base + threadIdx.x;
    if (i >= n || n < 2) return;
    if (sort_timed_out(status)) return;  // the pieces are not sorted: no tree to refit
    const uint32_t block_end = min(n, base + (uint32_t)kSplitRefitBlock);
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
    uint32_t child = i;  // (the leaf box is published by the first arrival's release)
    uint32_t p = parents_leaf[i];
    // at most n - 1 nodes on any walk (each node lets one arriver continue)
    for (uint32_t steps = 0; p != CPT_INVALID_INDEX; ++steps) {
        if (p >= n - 1 || steps >= n - 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }
        float* node = nodes + 24 * (size_t)p;
        const float4 meta = *reinterpret_cast<const float4*>(node + 20);  // Node word, right child, range end
        const uint32_t word = __float_as_uint(meta.x);
        const uint32_t left = word >> 2;
        const int side = left == child ? 0 : 1;
        const uint32_t j = __float_as_uint(meta.z);
        const bool local = min(p, j) >= base && max(p, j) < block_end;
        store_slot(node, side, slot);
        const uint32_t sib = left + (uint32_t)(1 - side);
        Box sb;
        if (local) {
            const uint32_t k = p - base;
            float* mine = s_box[2 * k + side];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) { mine[ax] = box.mn[ax]; mine[3 + ax] = box.mx[ax]; }
            __threadfence_block();
            const int arrived = atomicAdd(&s_count[k], 1);
            if (arrived == 0) return;
            if (arrived != 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }
            __threadfence_block();
            const volatile float* other = s_box[2 * k + (1 - side)];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) { sb.mn[ax] = other[ax]; sb.mx[ax] = other[3 + ax]; }
        } else {
            const int arrived = arrive_acq_rel(&counters[p]);
            if (arrived == 0) return;
            if (arrived != 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }
            const bool sib_internal = (word >> (1 - side)) & 1u;
            if (sib_internal) {
                const float2* q = reinterpret_cast<const float2*>(node_boxes + sib);
                const float2 x0 = __ldcg(q), x1 = __ldcg(q + 1), x2 = __ldcg(q + 2);
                sb.mn[0] = x0.x; sb.mn[1] = x0.y; sb.mn[2] = x1.x; sb.mx[0] = x1.y; sb.mx[1] = x2.x; sb.mx[2] = x2.y;
            } else {
                sb = piece_box(leaf_boxes, sib, true);
            }
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

// ---------------------------------------------------------------------------
// Treelet restructuring (CPT_SPLIT_TREELET; Karras and Aila, "Fast Parallel
// Construction of High-Quality Bounding Volume Hierarchies", HPG 2013), applied to
// the split tree after its refit. The cost of a tree is the sum of the surface
// areas of its internal nodes (the surface-area heuristic with the leaves fixed:
// every piece stays one leaf). A bottom-up walk with the refit's arrival counters
// reaches a node once both its subtrees are final; where the node has at least
// gamma leaves, its warp forms a treelet — the node's two children, then, up to 7
// leaves, the internal treelet leaf of largest area replaced by its two children —
// and finds the least-cost topology over those leaves by dynamic programming over
// their subsets, c(S) = area(S) + min over splits S = P + (S \ P) of c(P) + c(S \ P)
// (one leaf: 0), the lanes sharing out the 966 (subset, split) pairs of 7 leaves.
// A cheaper topology that is no taller than the old one replaces it in the same
// nodes (the treelet root keeps its index, box and parent). The result does not
// depend on timing: a treelet sees only its finished subtree, areas and sums are
// rounded without contraction, and equal costs go to the smallest split mask.
// One round with gamma = 4 (treelets of 4 to 6 leaves where a subtree has fewer
// than 7): on the C2 scene more rounds (gamma doubling) lower the binary tree's cost
// a little further but raise the node visits of the 8-wide tree collapsed from it.
// Since no treelet grows taller, the tree is never taller than the Karras tree it
// starts from.
// ---------------------------------------------------------------------------
constexpr int kTreeletBlock = 128;
constexpr int kTreeletWarps = kTreeletBlock / 32;
constexpr int kTreeletLeaves = 7;
constexpr int kTreeletSubsets = 1 << kTreeletLeaves;
constexpr int kTreeletPairs = 966;  // sum over k = 2..7 of C(7, k) (2^(k-1) - 1)
#ifndef CPT_TREELET_ROUNDS
#define CPT_TREELET_ROUNDS 1
#endif
#ifndef CPT_TREELET_GAMMA
#define CPT_TREELET_GAMMA 4
#endif
#ifndef CPT_TREELET_GAMMA_SHIFT
#define CPT_TREELET_GAMMA_SHIFT 1  // gamma doubles every round
#endif
constexpr int kTreeletRounds = CPT_TREELET_ROUNDS;
constexpr int kTreeletGamma = CPT_TREELET_GAMMA;
constexpr int kTreeletMaxLevels = 1024;

// Index of the first (subset, split) pair of the subsets of k leaves (k = 2..7;
// k = 8 gives the total).
__device__ __forceinline__ int treelet_class_start(int k)
{
    switch (k) {
    case 2: return 0;
    case 3: return 21;
    case 4: return 126;
    case 5: return 371;
    case 6: return 686;
    case 7: return 903;
    default: return kTreeletPairs;
    }
}

// Half the surface area of a box (lo xyz, hi xyz), rounded alike on every run.
__device__ __forceinline__ float half_area(const float* b)
{
    const float dx = __fsub_rn(b[3], b[0]), dy = __fsub_rn(b[4], b[1]), dz = __fsub_rn(b[5], b[2]);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

// A treelet as formed: its leaves and internal nodes.
struct TreeletForm {
    float box[kTreeletLeaves][6];
    uint32_t id[kTreeletLeaves];      // internal node index, or piece position for a leaf
    uint32_t height[kTreeletLeaves];
    uint32_t size[kTreeletLeaves];
    uint32_t from[kTreeletLeaves];    // parent * 2 + side: the record slot holding the leaf
    uint32_t inode[kTreeletLeaves - 1];  // the treelet's internal nodes, [0] = its root
    uint32_t internal_mask;           // bit k: treelet leaf k is an internal node
    uint32_t m;                       // treelet leaves (0: bad index met)
    float old_cost;                   // summed area of the treelet's internal nodes
};

struct TreeletWarp {
    TreeletForm form;
    float c[kTreeletSubsets];         // least cost over a subset (its area until its size class is done)
    float slot[kTreeletLeaves][10];   // the leaves' 40-B child slots, read before any rewrite
    uint8_t split[kTreeletSubsets];
};

// Treelet leaves k0 and k1 := the two children of internal node q. False on an out-of-range index.
__device__ bool treelet_take_children(const float* __restrict__ nodes, const float4* __restrict__ leaf_boxes,
                                      const uint2* __restrict__ info, uint32_t n, uint32_t q, int k0, int k1,
                                      TreeletForm& f)
{
    const float* rec = nodes + 24 * (size_t)q;
    const float4 meta = __ldcg(reinterpret_cast<const float4*>(rec + 20));
    const uint32_t word = __float_as_uint(meta.x);
    const uint32_t ids[2] = {word >> 2, __float_as_uint(meta.y)};
    for (int side = 0; side < 2; ++side) {
        const int k = side ? k1 : k0;
        const bool internal = (word >> side) & 1u;
        const uint32_t id = ids[side];
        if (internal ? id >= n - 1 : id >= n) return false;
        if (internal) {  // an internal child's slot starts with its box
            const float2* sp = reinterpret_cast<const float2*>(rec + 10 * side);
            const float2 a = __ldcg(sp), b = __ldcg(sp + 1), c = __ldcg(sp + 2);
            f.box[k][0] = a.x; f.box[k][1] = a.y; f.box[k][2] = b.x;
            f.box[k][3] = b.y; f.box[k][4] = c.x; f.box[k][5] = c.y;
            const uint2 g = __ldcg(info + id);
            f.size[k] = g.x;
            f.height[k] = g.y;
            f.internal_mask |= 1u << k;
        } else {
            const float4 lo = leaf_boxes[2 * (size_t)id], hi = leaf_boxes[2 * (size_t)id + 1];
            f.box[k][0] = lo.x; f.box[k][1] = lo.y; f.box[k][2] = lo.z;
            f.box[k][3] = hi.x; f.box[k][4] = hi.y; f.box[k][5] = hi.z;
            f.size[k] = 1;
            f.height[k] = 0;
            f.internal_mask &= ~(1u << k);
        }
        f.id[k] = id;
        f.from[k] = 2u * q + (uint32_t)side;
    }
    return true;
}

// Forms the treelet rooted at internal node r (one lane).
__device__ void treelet_form(const float* __restrict__ nodes, const float4* __restrict__ leaf_boxes,
                             const uint2* __restrict__ info, uint32_t n, uint32_t r, TreeletForm& f,
                             uint32_t* __restrict__ status)
{
    f.internal_mask = 0;
    f.inode[0] = r;
    bool ok = treelet_take_children(nodes, leaf_boxes, info, n, r, 0, 1, f);
    uint32_t m = 2, ni = 1;
    float old = 0.f;
    if (ok) {
        float rb[6];
        for (int a = 0; a < 3; ++a) {
            rb[a] = fminf(f.box[0][a], f.box[1][a]);
            rb[3 + a] = fmaxf(f.box[0][3 + a], f.box[1][3 + a]);
        }
        old = half_area(rb);
    }
    while (ok && m < (uint32_t)kTreeletLeaves) {
        int b = -1;
        float ba = -1.f;
        for (uint32_t k = 0; k < m; ++k)
            if ((f.internal_mask >> k) & 1u) {
                const float a = half_area(f.box[k]);
                if (a > ba) { ba = a; b = (int)k; }
            }
        if (b < 0) break;
        f.inode[ni++] = f.id[b];
        old = __fadd_rn(old, ba);
        ok = treelet_take_children(nodes, leaf_boxes, info, n, f.id[b], b, (int)m, f);
        ++m;
    }
    if (!ok) atomicOr(status, CPT_STATUS_BAD_INDEX);
    f.m = ok ? m : 0u;
    f.old_cost = old;
}

// Solves the warp's formed treelet (rooted at a node whose subtree is h_before tall)
// and rewrites it if cheaper and no taller; called by the whole warp.
__device__ void treelet_solve(float* __restrict__ nodes, uint32_t* __restrict__ parents_leaf,
                              uint32_t* __restrict__ parents_internal, uint2* __restrict__ info,
                              uint32_t h_before, const uint16_t* __restrict__ pairs, TreeletWarp& w)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();  // the form is written
    const TreeletForm& f = w.form;
    const uint32_t m = f.m;
    if (m < 3) {
        __syncwarp();  // every lane has read m before the next form is written
        return;
    }
    const uint32_t full = (1u << m) - 1u;
    if ((uint32_t)lane < m) {
        const uint32_t from = f.from[lane];
        const float2* sp = reinterpret_cast<const float2*>(nodes + 24 * (size_t)(from >> 1) + 10 * (from & 1u));
        for (int j = 0; j < 5; ++j) {
            const float2 v = __ldcg(sp + j);
            w.slot[lane][2 * j] = v.x;
            w.slot[lane][2 * j + 1] = v.y;
        }
    }
    for (uint32_t S = (uint32_t)lane + 1u; S <= full; S += 32u) {
        if (__popc(S) == 1) { w.c[S] = 0.f; continue; }
        float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
#pragma unroll
        for (int k = 0; k < kTreeletLeaves; ++k)
            if ((S >> k) & 1u)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    b[a] = fminf(b[a], f.box[k][a]);
                    b[3 + a] = fmaxf(b[3 + a], f.box[k][3 + a]);
                }
        w.c[S] = half_area(b);
    }
    __syncwarp();
    // size class k: C(7, k) subsets of 2^(k-1) - 1 splits each; a lane takes a subset,
    // or (k = 6, 7) a group of g lanes shares a subset's splits and reduces by shuffles.
    // The least (cost bits, split mask) wins.
    for (int k = 2; k <= (int)m; ++k) {
        const int subsets = k == 2 ? 21 : k == 3 ? 35 : k == 4 ? 35 : k == 5 ? 21 : k == 6 ? 7 : 1;
        const int g = k == 6 ? 4 : k == 7 ? 32 : 1;
        const int np = (1 << (k - 1)) - 1;
        const uint16_t* cls = pairs + treelet_class_start(k);
        for (int i0 = 0; i0 < subsets * g; i0 += 32) {
            const int idx = i0 + lane, rho = idx / g, q = idx % g;
            unsigned long long key = ~0ull;
            uint32_t S = 0;
            if (rho < subsets) {
                const uint16_t* ps = cls + rho * np;
                S = ps[0] & 127u;
                if (!(S & ~full))
                    for (int j = q; j < np; j += g) {
                        const uint32_t P = (uint32_t)ps[j] >> 7;
                        const float v = __fadd_rn(w.c[P], w.c[S ^ P]);
                        const unsigned long long kk = ((unsigned long long)__float_as_uint(v) << 32) | P;
                        key = kk < key ? kk : key;
                    }
            }
            for (int o = 1; o < g; o <<= 1) {
                const unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, key, o);
                key = other < key ? other : key;
            }
            if (rho < subsets && q == 0 && !(S & ~full)) {
                w.c[S] = __fadd_rn(w.c[S], __uint_as_float((uint32_t)(key >> 32)));
                w.split[S] = (uint8_t)(key & 127u);
            }
        }
        __syncwarp();
    }
    if (lane == 0 && w.c[full] < __fmul_rn(f.old_cost, 0.999999f)) {
        // the new topology, top-down: node j covers subset sub[j]; a child reference
        // is a treelet leaf k (< 8) or node 8 + j
        uint32_t sub[kTreeletLeaves - 1], ck[kTreeletLeaves - 1][2];
        uint32_t cnt = 1;
        sub[0] = full;
        bool ok = true;
        for (uint32_t j = 0; j < cnt && ok; ++j) {
            const uint32_t S = sub[j], P = w.split[S];
            const uint32_t X[2] = {P, S ^ P};
            for (int side = 0; side < 2; ++side) {
                if (X[side] == 0u || (X[side] & ~S)) { ok = false; break; }
                if (__popc(X[side]) == 1) {
                    ck[j][side] = (uint32_t)(__ffs(X[side]) - 1);
                } else {
                    if (cnt >= m - 1) { ok = false; break; }
                    sub[cnt] = X[side];
                    ck[j][side] = 8u + cnt;
                    ++cnt;
                }
            }
        }
        if (ok && cnt == m - 1) {
            uint32_t h[kTreeletLeaves - 1], sz[kTreeletLeaves - 1];
            for (int j = (int)cnt - 1; j >= 0; --j) {
                uint32_t hh = 0, ss = 0;
                for (int side = 0; side < 2; ++side) {
                    const uint32_t c = ck[j][side];
                    hh = max(hh, c < 8u ? f.height[c] : h[c - 8u]);
                    ss += c < 8u ? f.size[c] : sz[c - 8u];
                }
                h[j] = hh + 1u;
                sz[j] = ss;
            }
            if (h[0] <= h_before) {
                for (uint32_t j = 0; j < cnt; ++j) {
                    const uint32_t nd = f.inode[j];
                    float* rec = nodes + 24 * (size_t)nd;
                    uint32_t ids[2], word = 0;
                    for (int side = 0; side < 2; ++side) {
                        const uint32_t c = ck[j][side];
                        float slot[10];
                        if (c < 8u) {
                            ids[side] = f.id[c];
                            for (int a = 0; a < 10; ++a) slot[a] = w.slot[c][a];
                            if ((f.internal_mask >> c) & 1u) {
                                word |= 1u << side;
                                parents_internal[ids[side]] = nd;
                            } else {
                                parents_leaf[ids[side]] = nd;
                            }
                        } else {
                            const uint32_t x = c - 8u, X = sub[x];
                            ids[side] = f.inode[x];
                            word |= 1u << side;
                            for (int a = 0; a < 3; ++a) { slot[a] = FLT_MAX; slot[3 + a] = -FLT_MAX; }
                            for (uint32_t k = 0; k < m; ++k)
                                if ((X >> k) & 1u)
                                    for (int a = 0; a < 3; ++a) {
                                        slot[a] = fminf(slot[a], f.box[k][a]);
                                        slot[3 + a] = fmaxf(slot[3 + a], f.box[k][3 + a]);
                                    }
                            slot[6] = slot[7] = slot[8] = slot[9] = 0.0f;
                            parents_internal[ids[side]] = nd;
                        }
                        store_slot(rec, side, slot);
                    }
                    word |= ids[0] << 2;
                    reinterpret_cast<float4*>(rec)[5] =
                        make_float4(__uint_as_float(word), __uint_as_float(ids[1]), 0.f, 0.f);
                    info[nd] = make_uint2(sz[j], h[j]);
                }
            }
        }
        __threadfence();
    }
    __syncwarp();
}

// A round of treelet restructuring over the split tree: every piece's walker goes
// up; the second arrival at a node records its size and height and, at gamma or
// more leaves, has its warp form and solve the node's treelet.
__global__ void __launch_bounds__(kTreeletBlock) k_treelet(const uint32_t* __restrict__ n_pieces,
                                                          float* __restrict__ nodes,
                                                          const float4* __restrict__ leaf_boxes,
                                                          uint32_t* __restrict__ parents_leaf,
                                                          uint32_t* __restrict__ parents_internal,
                                                          int* __restrict__ counters, uint2* __restrict__ info,
                                                          uint32_t gamma, uint32_t* __restrict__ status)
{
    // (subset, split) pairs by subset size: a subset S of k >= 2 leaves lists its
    // 2^(k-1) - 1 splits P (P holds S's lowest leaf, P != S) from
    // treelet_class_start(k) + rank of S among the k-leaf subsets x (2^(k-1) - 1).
    __shared__ uint16_t s_pairs[kTreeletPairs];
    __shared__ TreeletWarp s_warp[kTreeletWarps];
    if (threadIdx.x < kTreeletSubsets) {
        const uint32_t S = threadIdx.x;
        const int k = __popc(S);
        if (k >= 2) {
            uint32_t rank = 0;
            for (uint32_t x = 1; x < S; ++x) rank += __popc(x) == k ? 1u : 0u;
            const uint32_t np = (1u << (k - 1)) - 1u, low = S & (0u - S), rest = S ^ low;
            uint16_t* out = s_pairs + treelet_class_start(k) + rank * np;
            for (uint32_t j = 0; j < np; ++j) {
                uint32_t P = low, bits = rest, jj = j;
                while (bits) {
                    const uint32_t b = bits & (0u - bits);
                    if (jj & 1u) P |= b;
                    jj >>= 1;
                    bits ^= b;
                }
                out[j] = (uint16_t)(S | (P << 7));
            }
        }
    }
    __syncthreads();
    const uint32_t n = *n_pieces;
    if (n < 3) return;
    if (sort_timed_out(status)) return;  // (uniform over the launch: set before it started)
    const int lane = threadIdx.x & 31;
    TreeletWarp& w = s_warp[threadIdx.x >> 5];
    const uint32_t i = blockIdx.x * kTreeletBlock + threadIdx.x;
    bool active = i < n;
    uint32_t node = active ? parents_leaf[i] : CPT_INVALID_INDEX;
    uint32_t height = 0;
    for (int level = 0; __any_sync(0xFFFFFFFFu, active); ++level) {
        bool process = false;
        if (active) {
            if (node == CPT_INVALID_INDEX) {
                active = false;  // passed the root
            } else if (node >= n - 1 || level >= kTreeletMaxLevels) {
                atomicOr(status, CPT_STATUS_BAD_INDEX);
                active = false;
            } else {
                const int arrived = arrive_acq_rel(&counters[node]);
                if (arrived != 1) {
                    if (arrived != 0) atomicOr(status, CPT_STATUS_BAD_INDEX);
                    active = false;
                } else {
                    const float4 meta = __ldcg(reinterpret_cast<const float4*>(nodes + 24 * (size_t)node + 20));
                    const uint32_t word = __float_as_uint(meta.x);
                    const uint32_t ids[2] = {word >> 2, __float_as_uint(meta.y)};
                    uint32_t size = 0;
                    bool ok = true;
                    height = 0;
                    for (int side = 0; side < 2; ++side) {
                        if ((word >> side) & 1u) {
                            if (ids[side] >= n - 1) { ok = false; continue; }
                            const uint2 g = __ldcg(info + ids[side]);
                            size += g.x;
                            height = max(height, g.y);
                        } else {
                            if (ids[side] >= n) ok = false;
                            size += 1u;
                        }
                    }
                    if (!ok) {
                        atomicOr(status, CPT_STATUS_BAD_INDEX);
                        active = false;
                    } else {
                        height += 1u;
                        info[node] = make_uint2(size, height);
                        process = size >= gamma;
                    }
                }
            }
        }
        uint32_t todo = __ballot_sync(0xFFFFFFFFu, process);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1u;
            const uint32_t r = __shfl_sync(0xFFFFFFFFu, node, src);
            const uint32_t hr = __shfl_sync(0xFFFFFFFFu, height, src);
            if (lane == 0) treelet_form(nodes, leaf_boxes, info, n, r, w.form, status);
            treelet_solve(nodes, parents_leaf, parents_internal, info, hr, s_pairs, w);
        }
        if (active) node = __ldcg(parents_internal + node);
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
    uint2* info;  // treelet restructuring: per internal node (leaves, height)
};

template <typename K>
size_t split_layout(uint32_t n, uint32_t cap, bool treelet, void* base, SplitScratch<K>* out)
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
    s.info = treelet ? c.take<uint2>(cap) : nullptr;
    if (out) *out = s;
    return c.used();
}

inline uint64_t split_capacity(uint32_t n, float extra_ratio)
{
    const double r = extra_ratio > 0.f ? (double)extra_ratio : 0.0;
    return (uint64_t)n + (uint64_t)floor(r * (double)n);
}

template <typename K>
int split_impl(cpt_bvh* bvh, uint32_t cap, bool treelet, void* nodes, void* scratch,
               cudaStream_t stream)
{
    constexpr int P = KeyTraits<K>::passes;
    const uint32_t n = bvh->n;
    SplitScratch<K> s;
    split_layout<K>(n, cap, treelet, scratch, &s);
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
    k_split_first<<<ctiles, kSplitBlock, 0, stream>>>(n, s.counts, s.tile_sums);
    CPT_LAUNCH_CHECK();
    const uint32_t eblocks = (uint32_t)(((uint64_t)cap + (uint64_t)kSplitBlock * kEmitPieces - 1) /
                                        ((uint64_t)kSplitBlock * kEmitPieces));
    k_split_emit<K><<<eblocks, kSplitBlock, 0, stream>>>(bvh->tris, n, s.counts, s.n_pieces, bvh->node_boxes,
                                                         s.pieces, s.keys[0], s.hist, s.zero, s.zero_words);
    CPT_LAUNCH_CHECK();
    k_scan_offsets<<<P, kRadix, 0, stream>>>(s.hist, s.offsets);
    CPT_LAUNCH_CHECK();
    const uint32_t tiles = (cap + kSortTile - 1) / kSortTile;
    uint32_t* lookback = s.zero + 32;
    const K* keys;
    if constexpr (sizeof(K) == 8) {  // as 32-bit halves: the sorted keys end in keys[1]
        if (const int rc = onesweep_sort64_halves(reinterpret_cast<const uint64_t*>(s.keys[0]),
                                                  reinterpret_cast<uint64_t*>(s.keys[1]), cap, 0, s.n_pieces, s.vals,
                                                  s.offsets, lookback, s.zero, bvh->status, SortWait(), true, false,
                                                  stream))
            return rc;
        keys = s.keys[1];
    } else {
        const size_t smem = onesweep_smem<K>();
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
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
        keys = s.keys[P & 1];
    }
    const uint32_t* order = s.vals[(P - 1) & 1];
    k_topology<K><<<(cap + 255) / 256, 256, 0, stream>>>(keys, 0, s.n_pieces, s.children, s.parents_leaf,
                                                          s.parents_internal, s.counters, static_cast<float4*>(nodes),
                                                          bvh->status, cap - 1);
    CPT_LAUNCH_CHECK();
    k_split_refit<<<(cap + kSplitRefitBlock - 1) / kSplitRefitBlock, kSplitRefitBlock, 0, stream>>>(
        bvh->tris, s.pieces, order, s.n_pieces, s.children,
                                                          s.parents_leaf, s.parents_internal, s.counters,
                                                          static_cast<float*>(nodes), s.node_boxes, s.leaf_boxes, n,
                                                          bvh->status);
    CPT_LAUNCH_CHECK();
    if (treelet) {
        for (int round = 0; round < kTreeletRounds; ++round) {
            CPT_CUDA_TRY(cudaMemsetAsync(s.counters, 0, sizeof(int) * (size_t)cap, stream));
            k_treelet<<<(cap + kTreeletBlock - 1) / kTreeletBlock, kTreeletBlock, 0, stream>>>(
                s.n_pieces, static_cast<float*>(nodes), s.leaf_boxes, s.parents_leaf, s.parents_internal, s.counters,
                s.info, (uint32_t)kTreeletGamma << (CPT_TREELET_GAMMA_SHIFT * round), bvh->status);
            CPT_LAUNCH_CHECK();
        }
    }
    return CPT_OK;
}

}  // namespace
}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_lbvh_split_bytes(uint32_t n, int morton_bits, float extra_ratio, uint32_t flags,
                                       size_t* node_bytes)
{
    if (n < 2 || n > kMaxTriangles || (morton_bits != 30 && morton_bits != 63)) return 0;
    if (!(extra_ratio >= 0.f) || !(extra_ratio <= 64.f)) return 0;  // the range cpt_lbvh_split accepts
    const bool treelet = flags & CPT_SPLIT_TREELET;
    if (flags & ~CPT_SPLIT_TREELET) return 0;
    const uint64_t cap = split_capacity(n, extra_ratio);
    if (cap >= (1ull << 31)) return 0;
    if (node_bytes) *node_bytes = align_up((size_t)(cap - 1) * 96, 256);
    return morton_bits == 30 ? split_layout<uint32_t>(n, (uint32_t)cap, treelet, nullptr, nullptr)
                             : split_layout<uint64_t>(n, (uint32_t)cap, treelet, nullptr, nullptr);
}

extern "C" int cpt_lbvh_split(cpt_bvh* bvh, float extra_ratio, uint32_t flags, void* nodes, size_t node_bytes,
                              void* scratch, size_t scratch_bytes, cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_split");
    if (!bvh || !bvh->tris || !bvh->node_boxes || !bvh->status || !nodes || !scratch) return CPT_ERR_INVALID_ARGUMENT;
    if (!(extra_ratio >= 0.f) || !(extra_ratio <= 64.f)) return CPT_ERR_INVALID_ARGUMENT;
    size_t nb = 0;
    const size_t need = cpt_lbvh_split_bytes(bvh->n, bvh->morton_bits, extra_ratio, flags, &nb);
    if (!need) return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < need || node_bytes < nb) return CPT_ERR_SCRATCH_TOO_SMALL;
    if ((reinterpret_cast<uintptr_t>(nodes) & 15) || (reinterpret_cast<uintptr_t>(scratch) & 255))
        return CPT_ERR_INVALID_ARGUMENT;
    const uint32_t cap = (uint32_t)split_capacity(bvh->n, extra_ratio);
    const bool treelet = flags & CPT_SPLIT_TREELET;
    const int rc = bvh->morton_bits == 30 ? split_impl<uint32_t>(bvh, cap, treelet, nodes, scratch, stream)
                                          : split_impl<uint64_t>(bvh, cap, treelet, nodes, scratch, stream);
    if (rc) return rc;
    bvh->split_nodes = nodes;
    bvh->split_capacity = cap;
    bvh->wide_nodes = nullptr;  // a wide tree of the previous binary tree is stale
    bvh->wide_tris = nullptr;
    bvh->wide_capacity = 0;
    return CPT_OK;
}
