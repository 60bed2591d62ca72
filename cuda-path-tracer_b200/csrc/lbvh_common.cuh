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

template <typename K>
__global__ void __launch_bounds__(256) k_topology(const K* __restrict__ keys, uint32_t n_arg,
                                                  const uint32_t* __restrict__ n_ptr, uint32_t* __restrict__ children,
                                                  uint32_t* __restrict__ parents_leaf,
                                                  uint32_t* __restrict__ parents_internal, int* __restrict__ counters,
                                                  float4* __restrict__ nodes, const uint32_t* __restrict__ status)
{
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int nn = (int)(n_ptr ? *n_ptr : n_arg);
    if (i >= nn - 1) return;
    if (sort_timed_out(status)) return;  // the keys are not sorted: build nothing from them
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

}  // namespace cpt
