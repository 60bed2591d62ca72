// Pieces of the LBVH build shared by the reference-format build (lbvh.cu) and
// the split traversal BVH (split.cu): key traits and Morton helpers, the Karras
// topology kernel, box helpers and the 40-B traversal child slot.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "cpt.h"
#include "cpt_device.cuh"

namespace cpt {

template <typename K> struct KeyTraits;
template <> struct KeyTraits<uint32_t> { static constexpr int passes = 4, order = 10, total_bits = 32; };
template <> struct KeyTraits<uint64_t> { static constexpr int passes = 8, order = 21, total_bits = 64; };

// Bit spreading for the 3-D interleave (x -> bit 3i, y -> 3i+1, z -> 3i+2, the
// layout of morton.h:63-102): the standard shift-and-mask "part 1 by 2" sequence
// on 64 bits, valid for inputs of up to 21 bits.
__device__ __forceinline__ uint64_t spread3(uint32_t v)
{
    uint64_t x = v & 0x1FFFFFull;
    x = (x | (x << 32)) & 0x001F00000000FFFFull;
    x = (x | (x << 16)) & 0x001F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// quantize (math_util.h:10-13): clamp(int(x * n), 0, n - 1); cvt.rzi saturates and maps NaN to 0.
__device__ __forceinline__ uint32_t quantize(float x, uint32_t n)
{
    int32_t q = __float2int_rz(__fmul_rn(x, (float)n));
    int32_t hi = (int32_t)(n - 1);
    q = q < hi ? q : hi;
    return (uint32_t)(q > 0 ? q : 0);
}

struct Box { float mn[3], mx[3]; };

// True when a sort pass of this build gave up a look-back wait (CPT_STATUS_TIMEOUT):
// the kernels after the sort then return at once, leaving their outputs unwritten,
// and the build reports CPT_ERR_DEVICE_TIMEOUT. The status word is only read here,
// in kernels launched after the sort, so the kernel boundary orders it.
__device__ __forceinline__ bool sort_timed_out(const uint32_t* status)
{
    return (__ldcg(status) & CPT_STATUS_TIMEOUT) != 0u;
}

// ---------------------------------------------------------------------------
// Karras radix tree over the sorted keys (BVHBuilder.cu:107-201). Also writes
// the Node word into the traversal record, zeroes the refit counters and marks
// the root's parent. The leaf count is n_arg, or *n_ptr when n_ptr is set (a
// count known only on the device; the grid then covers the largest count).
// ---------------------------------------------------------------------------
template <typename K>
__device__ __forceinline__ int key_delta(const K* __restrict__ keys, K ki, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    K kj = __ldg(keys + j);
    if (ki == kj) return __clz(i ^ j) + KeyTraits<K>::total_bits;
    if (sizeof(K) == 8) return __clzll((long long)(ki ^ kj));
    return __clz((int)(ki ^ kj));
}

// Internal node i of the radix tree over nn sorted keys: its Node word, the parents of
// its two children, its traversal record's Node word / right index / range end, and
// its refit counter (zeroed).
template <typename K>
__device__ __forceinline__ void topology_node(const K* __restrict__ keys, int nn, int i, uint32_t* __restrict__ children,
                                              uint32_t* __restrict__ parents_leaf,
                                              uint32_t* __restrict__ parents_internal, int* __restrict__ counters,
                                              float4* __restrict__ nodes)
{
    const K ki = keys[i];
    int dd = key_delta(keys, ki, nn, i, i + 1) - key_delta(keys, ki, nn, i, i - 1);
    int d = (dd > 0) - (dd < 0);
    int dmin = key_delta(keys, ki, nn, i, i - d);
    int lmax = 2;
    while (key_delta(keys, ki, nn, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    while (lmax > 1) {
        lmax /= 2;
        if (key_delta(keys, ki, nn, i, i + (l + lmax) * d) > dmin) l += lmax;
    }
    const int j = i + l * d;
    const int dnode = key_delta(keys, ki, nn, i, j);
    int s = 0;
    while (l > 1) {
        l = (l + 1) / 2;
        if (key_delta(keys, ki, nn, i, i + (s + l) * d) > dnode) s += l;
    }
    s = i + s * d + (d < 0 ? d : 0);
    uint32_t type = 0;
    if (min(i, j) != s) { type |= 1u; parents_internal[s] = (uint32_t)i; }
    else parents_leaf[s] = (uint32_t)i;
    if (max(i, j) != s + 1) { type |= 2u; parents_internal[s + 1] = (uint32_t)i; }
    else parents_leaf[s + 1] = (uint32_t)i;
    const uint32_t word = ((uint32_t)s << 2) | type;
    children[i] = word;
    // Node word, the right child's index (s + 1 here; any index in trees whose siblings
    // are not adjacent), and j, the other end of the node's leaf range [min(i, j), max(i, j)]
    nodes[6 * (size_t)i + 5] = make_float4(__uint_as_float(word), __uint_as_float((uint32_t)s + 1u),
                                           __uint_as_float((uint32_t)j), 0.0f);
    counters[i] = 0;
    if (i == 0) parents_internal[0] = CPT_INVALID_INDEX;
}

// Node word of a traversal record past the tree's last internal node (a tree over fewer
// leaves than its arrays hold, the split tree): no valid node word has both type bits and
// an all-ones left index.
constexpr uint32_t kUnusedNode = 0xFFFFFFFFu;

// node_cap: the internal-node records of `nodes`; those past the tree get kUnusedNode.
template <typename K>
__global__ void __launch_bounds__(256) k_topology(const K* __restrict__ keys, uint32_t n_arg,
                                                  const uint32_t* __restrict__ n_ptr, uint32_t* __restrict__ children,
                                                  uint32_t* __restrict__ parents_leaf,
                                                  uint32_t* __restrict__ parents_internal, int* __restrict__ counters,
                                                  float4* __restrict__ nodes, const uint32_t* __restrict__ status,
                                                  uint32_t node_cap)
{
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int nn = (int)(n_ptr ? *n_ptr : n_arg);
    if (i >= nn - 1) {
        if ((uint32_t)i < node_cap) nodes[6 * (size_t)i + 5] = make_float4(__uint_as_float(kUnusedNode), 0.f, 0.f, 0.f);
        return;
    }
    if (sort_timed_out(status)) return;  // the keys are not sorted: build nothing from them
    topology_node(keys, nn, i, children, parents_leaf, parents_internal, counters, nodes);
}

// 40-B slot at float offset 10*side of a 96-B node; 8-B aligned float2 stores.
__device__ __forceinline__ void store_slot(float* node, int side, const float s[10])
{
    float2* p = reinterpret_cast<float2*>(node + 10 * side);
#pragma unroll
    for (int k = 0; k < 5; ++k) p[k] = make_float2(s[2 * k], s[2 * k + 1]);
}

__device__ __forceinline__ Box leaf_box(const float v[9])
{
    Box b;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        float mn = FLT_MAX, mx = -FLT_MAX;
#pragma unroll
        for (int vv = 0; vv < 3; ++vv) { mn = gmin(mn, v[3 * vv + ax]); mx = gmax(mx, v[3 * vv + ax]); }
        b.mn[ax] = mn;
        b.mx[ax] = mx;
    }
    return b;
}


// Refit arrival counter: one atomic increment that releases this thread's earlier
// stores (its child slot and box) and acquires those of the thread that came before
// it at the same parent (the sibling's box), device-wide.
__device__ __forceinline__ int arrive_acq_rel(int* counter)
{
#ifdef CPT_REFIT_FENCES
    __threadfence();
    const int r = atomicAdd(counter, 1);
    __threadfence();
    return r;
#else
    int r;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], 1;" : "=r"(r) : "l"(counter) : "memory");
    return r;
#endif
}

// Triangle permutation fused with the bottom-up refit, one leaf (shared by the single
// build's k_gather_refit and the batched k_batch_refit). Thread i gathers sorted
// triangle i (the 40-B reference record), computes its leaf box, then walks up. At each
// parent it writes its child slot of the parent's 96-B traversal node (the triangle for
// a leaf, the box for an internal node); the second child to arrive (atomic counter)
// reads its sibling's box — the box the sibling's thread computed, which for a leaf is
// the reference's box of the triangle's vertices (BVHBuilder.cu:73-80) — and stores
// left.unite(right). Below the nodes whose leaf range leaves the block, the counter and
// the sibling's box live in shared memory (block-scope fences order them); above, the
// counter increment is a global acquire-release atomic: it publishes this thread's slot
// and box stores and makes the sibling's visible to the second arriver (the
// reference's refit has no ordering between them, BVHBuilder.cu:63-86).
// The work of one leaf i (sorted position) in a block of leaves [base, block_end):
// gather triangle src of tris_in into tris_out[i], then the bottom-up walk. s_count /
// s_box are the block's shared arrival counters and first-arriver boxes (zeroed
// counters before the first walk).
__device__ __forceinline__ void gather_refit_leaf(const float* __restrict__ tris_in, uint32_t src, uint32_t i,
                                                  uint32_t n, uint32_t base, uint32_t block_end,
                                                  float* __restrict__ tris_out,
                                                  const uint32_t* __restrict__ parents_leaf,
                                                  const uint32_t* __restrict__ parents_internal,
                                                  int* __restrict__ counters, float* __restrict__ nodes,
                                                  cpt_bbox* __restrict__ node_boxes, uint32_t* __restrict__ status,
                                                  int* s_count, float (*s_box)[6])
{
    if (src >= n) {  // only after a failed sort pass (its status is already set): stay in bounds
        atomicOr(status, CPT_STATUS_BAD_INDEX);
        src = n - 1;
    }
    const float2* s2 = reinterpret_cast<const float2*>(tris_in + 10ull * src);
    const float2 a = __ldg(s2), b = __ldg(s2 + 1), c = __ldg(s2 + 2), d = __ldg(s2 + 3), e = __ldg(s2 + 4);
    float2* o2 = reinterpret_cast<float2*>(tris_out + 10ull * i);
    o2[0] = a; o2[1] = b; o2[2] = c; o2[3] = d; o2[4] = e;
    const float v[9] = {a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x};
    // leaf slot: v0, the leaf's index (the triangle a hit reports), v1 - v0, v2 - v0
    float slot[10] = {v[0], v[1], v[2], __uint_as_float(i),
                      __fsub_rn(v[3], v[0]), __fsub_rn(v[4], v[1]), __fsub_rn(v[5], v[2]),
                      __fsub_rn(v[6], v[0]), __fsub_rn(v[7], v[1]), __fsub_rn(v[8], v[2])};
    Box box = leaf_box(v);  // BVHBuilder.cu:73-74, BBox.cpp:26-30
    uint32_t child = i;
    uint32_t p = parents_leaf[i];
    // A node lets at most one arriver continue (the second; a third is refused), so
    // a walk passes at most n - 1 nodes even on a corrupt topology; the step count
    // makes that bound explicit.
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
            if (arrived != 1) { atomicOr(status, CPT_STATUS_BAD_INDEX); return; }  // a third visit: not a tree
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
                const float2* q = reinterpret_cast<const float2*>(tris_out + 10ull * sib);
                const float2 x0 = __ldcg(q), x1 = __ldcg(q + 1), x2 = __ldcg(q + 2), x3 = __ldcg(q + 3), x4 = __ldcg(q + 4);
                const float sv[9] = {x0.x, x0.y, x1.x, x1.y, x2.x, x2.y, x3.x, x3.y, x4.x};
                sb = leaf_box(sv);
            }
        }
        Box u;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float lmn = side == 0 ? box.mn[ax] : sb.mn[ax], rmn = side == 0 ? sb.mn[ax] : box.mn[ax];
            const float lmx = side == 0 ? box.mx[ax] : sb.mx[ax], rmx = side == 0 ? sb.mx[ax] : box.mx[ax];
            u.mn[ax] = gmin(lmn, rmn);
            u.mx[ax] = gmax(lmx, rmx);
        }
        box = u;
        float2* ob = reinterpret_cast<float2*>(node_boxes + p);
        ob[0] = make_float2(box.mn[0], box.mn[1]);
        ob[1] = make_float2(box.mn[2], box.mx[0]);
        ob[2] = make_float2(box.mx[1], box.mx[2]);
        // internal slot for the next level: the box, padded
#pragma unroll
        for (int k = 0; k < 3; ++k) { slot[k] = box.mn[k]; slot[3 + k] = box.mx[k]; }
        slot[6] = slot[7] = slot[8] = slot[9] = 0.0f;
        child = p;
        p = parents_internal[p];
    }
}

}  // namespace cpt
