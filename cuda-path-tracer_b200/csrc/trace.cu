// Ray queries against a built LBVH (cpt_trace): one thread per ray over a
// persistent grid, shared-memory node stack, 16-B vectorised record loads.
#include <cuda_runtime.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_internal.h"
#include "traverse.cuh"

namespace cpt {

constexpr int kTraceBlock = 128;

template <bool kAny, bool kStats>
__global__ void __launch_bounds__(kTraceBlock) k_trace(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                                                       const float4* __restrict__ rays, uint32_t n,
                                                       float4* __restrict__ hits, uint2* __restrict__ stats,
                                                       uint32_t* __restrict__ status)
{
    __shared__ uint32_t s_stack[CPT_TRAVERSAL_STACK * kTraceBlock];
    uint32_t* stack = s_stack + threadIdx.x;
    bool overflow = false;
    for (uint32_t i = blockIdx.x * kTraceBlock + threadIdx.x; i < n; i += gridDim.x * kTraceBlock) {
        const float4 ro = __ldg(rays + 2 * (size_t)i), rd = __ldg(rays + 2 * (size_t)i + 1);
        uint32_t nn = 0, nt = 0;
        Hit h = traverse<kAny, kTraceBlock, kStats>(nodes, tris, mk3(ro.x, ro.y, ro.z), mk3(rd.x, rd.y, rd.z), stack,
                                                    overflow, nn, nt);
        hits[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.tri));
        if (kStats) stats[i] = make_uint2(nn, nt);
    }
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
}

}  // namespace cpt

using namespace cpt;

extern "C" int cpt_trace(const cpt_bvh* bvh, const float* rays, uint32_t n, int any_hit, cpt_hit* hits,
                         uint32_t* stats, cudaStream_t stream)
{
    if (!bvh || !bvh->nodes || !bvh->tri_records || !bvh->status || (n && (!rays || !hits)))
        return CPT_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(rays) & 15) || (reinterpret_cast<uintptr_t>(hits) & 15))
        return CPT_ERR_INVALID_ARGUMENT;
    if (n == 0) return CPT_OK;
    const int blocks = (int)std::min<size_t>((n + kTraceBlock - 1) / kTraceBlock, (size_t)sm_count() * 16);
    const float4* nd = static_cast<const float4*>(bvh->nodes);
    const float4* tr = static_cast<const float4*>(bvh->tri_records);
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    float4* h4 = reinterpret_cast<float4*>(hits);
    uint2* st = reinterpret_cast<uint2*>(stats);
    CPT_PROF(K_TRACE, stream);
    if (any_hit) {
        if (stats) k_trace<true, true><<<blocks, kTraceBlock, 0, stream>>>(nd, tr, r4, n, h4, st, bvh->status);
        else k_trace<true, false><<<blocks, kTraceBlock, 0, stream>>>(nd, tr, r4, n, h4, st, bvh->status);
    } else {
        if (stats) k_trace<false, true><<<blocks, kTraceBlock, 0, stream>>>(nd, tr, r4, n, h4, st, bvh->status);
        else k_trace<false, false><<<blocks, kTraceBlock, 0, stream>>>(nd, tr, r4, n, h4, st, bvh->status);
    }
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}
