// Ray queries against a built LBVH, its split tree or its wide tree (cpt_trace):
// persistent warps over the ray array that refill their idle lanes from a shared
// pool, 96-B binary node or 80-B wide node loads, shared-memory node stack.
#include <cuda_runtime.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_internal.h"
#include "traverse.cuh"

namespace cpt {

constexpr int kTraceBlock = 128;
constexpr int kTraceSteps = 1024;

template <bool kAny, bool kStats>
__global__ void __launch_bounds__(kTraceBlock) k_trace(const float4* __restrict__ nodes, const float4* __restrict__ rays,
                                                       uint32_t n, float4* __restrict__ hits, uint2* __restrict__ stats,
                                                       uint32_t* __restrict__ pool, uint32_t* __restrict__ status,
                                                       uint32_t max_visits)
{
    __shared__ uint32_t s_stack[kSmemStack * kTraceBlock];
    bool overflow = false;
    uint32_t nn = 0, nt = 0;
    auto nodes_of = [&](uint32_t, uint32_t& mv) -> const float4* {  // one BVH for every ray
        mv = max_visits;
        return nodes;
    };
    persistent_trace_views<kAny, kTraceBlock, kStats, kTraceSteps>(nodes_of, rays, n, hits, pool, s_stack + threadIdx.x,
                                                                   overflow, nn, nt, nullptr, stats);
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
}

template <bool kAny, bool kStats>
__global__ void __launch_bounds__(kTraceBlock) k_trace_wide(const float4* __restrict__ nodes,
                                                            const float4* __restrict__ tris, uint32_t node_cap,
                                                            const float4* __restrict__ rays, uint32_t n,
                                                            float4* __restrict__ hits, uint2* __restrict__ stats,
                                                            uint32_t* __restrict__ pool, uint32_t* __restrict__ status)
{
    __shared__ uint2 s_stack[kWideSmemStack * kTraceBlock];
    bool overflow = false;
    uint32_t nn = 0, nt = 0;
    auto wide_of = [&](uint32_t, uint32_t& mv, const float4*& tr) -> const float4* {
        mv = node_cap;
        tr = tris;
        return nodes;
    };
    persistent_trace_wide<kAny, kTraceBlock, kStats, kTraceSteps, false>(
        wide_of, rays, n, pool, s_stack + threadIdx.x, overflow, nn, nt, nullptr,
        [&](uint32_t ray, const WideState& s) {
            hits[ray] = make_float4(s.best.t, s.best.u, s.best.v, __uint_as_float(s.best.tri));
            if (kStats && stats) stats[ray] = make_uint2(s.visits, s.tests);
        });
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
}

template <bool kAny, bool kStats>
int launch_trace_wide(const cpt_bvh* bvh, const float4* r4, uint32_t n, float4* h4, uint2* st, uint32_t* pool,
                      cudaStream_t stream)
{
    static int per_sm[2][2] = {{0, 0}, {0, 0}};
    int& occ = per_sm[kAny][kStats];
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trace_wide<kAny, kStats>, kTraceBlock, 0) !=
                cudaSuccess ||
            occ < 1)
            occ = 1;
    }
    const int blocks = (int)std::min<size_t>((n + kTraceBlock - 1) / kTraceBlock, (size_t)sm_count() * occ);
    k_trace_wide<kAny, kStats><<<blocks, kTraceBlock, 0, stream>>>(
        static_cast<const float4*>(bvh->wide_nodes), static_cast<const float4*>(bvh->wide_tris), bvh->wide_capacity - 1,
        r4, n, h4, st, pool, bvh->status);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

template <bool kAny, bool kStats>
int launch_trace(const float4* nd, const float4* r4, uint32_t n, float4* h4, uint2* st, uint32_t* pool,
                 uint32_t* status, uint32_t mv, cudaStream_t stream)
{
    static int per_sm[2][2] = {{0, 0}, {0, 0}};
    int& occ = per_sm[kAny][kStats];
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_trace<kAny, kStats>, kTraceBlock, 0) != cudaSuccess ||
            occ < 1)
            occ = 1;
    }
    const int blocks = (int)std::min<size_t>((n + kTraceBlock - 1) / kTraceBlock, (size_t)sm_count() * occ);
    k_trace<kAny, kStats><<<blocks, kTraceBlock, 0, stream>>>(nd, r4, n, h4, st, pool, status, mv);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

}  // namespace cpt

using namespace cpt;

extern "C" int cpt_trace(const cpt_bvh* bvh, const float* rays, uint32_t n, int any_hit, cpt_hit* hits,
                         uint32_t* stats, cudaStream_t stream)
{
    CPT_RANGE("cpt_trace");
    if (!bvh || !bvh->nodes || !bvh->status || (n && (!rays || !hits))) return CPT_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(rays) & 15) || (reinterpret_cast<uintptr_t>(hits) & 15))
        return CPT_ERR_INVALID_ARGUMENT;
    if (n == 0) return CPT_OK;
    // the split BVH when one was built (same hits, fewer node visits)
    const float4* nd = static_cast<const float4*>(bvh->split_nodes ? bvh->split_nodes : bvh->nodes);
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    float4* h4 = reinterpret_cast<float4*>(hits);
    uint2* st = reinterpret_cast<uint2*>(stats);
    uint32_t* pool = bvh->status + 1;  // ray pool counter of the persistent kernel
    CPT_CUDA_TRY(cudaMemsetAsync(pool, 0, sizeof(uint32_t), stream));
    // a ray fetches each internal node at most once
    const uint32_t mv = bvh->split_nodes ? (bvh->split_capacity | kFastSlabBit) : bvh->n;
    CPT_PROF(K_TRACE, stream);
    if (bvh->wide_nodes) {  // the wide tree when one was built
        if (any_hit) return stats ? launch_trace_wide<true, true>(bvh, r4, n, h4, st, pool, stream)
                                  : launch_trace_wide<true, false>(bvh, r4, n, h4, st, pool, stream);
        return stats ? launch_trace_wide<false, true>(bvh, r4, n, h4, st, pool, stream)
                     : launch_trace_wide<false, false>(bvh, r4, n, h4, st, pool, stream);
    }
    if (any_hit) return stats ? launch_trace<true, true>(nd, r4, n, h4, st, pool, bvh->status, mv, stream)
                              : launch_trace<true, false>(nd, r4, n, h4, st, pool, bvh->status, mv, stream);
    return stats ? launch_trace<false, true>(nd, r4, n, h4, st, pool, bvh->status, mv, stream)
                 : launch_trace<false, false>(nd, r4, n, h4, st, pool, bvh->status, mv, stream);
}
