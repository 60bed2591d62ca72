// Closest-hit / any-hit traversal over the compact LBVH records.
//
// Follows CUDA::trace (source/application/cuda/trace.h:73-169) decision for
// decision — both children tested (left first), both-farther-than-best pruning,
// nearer child first (ties to the left), the farther internal child pushed or
// the farther triangle recorded, a nearer triangle ending the descent — so the
// returned (t, triangle, u, v) are those of the reference, with the same
// Möller-Trumbore (intersection.h:28-59) and slab (intersection.h:106-117)
// arithmetic in round-to-nearest intrinsics.
//
// What changes is the memory side:
//  * one 64-B record per internal node holds both children's boxes and the Node
//    word (4 x 16-B loads), instead of a 4-B Node load followed by a 24-B box
//    load per internal child from a separate array;
//  * one 48-B record per triangle (v0 | info, v1 - v0, v2 - v0; 3 x 16-B loads)
//    instead of an unaligned 40-B record — the stored edges are the same
//    subtractions the test performs, so the bits are unchanged;
//  * 1/d is computed once per ray instead of per box (same value);
//  * the node stack lives in shared memory, one column per thread
//    (stack[depth * kBlock + thread]), CPT_TRAVERSAL_STACK deep like the
//    reference's 64-entry local array; a push beyond it is dropped and reported
//    (CPT_STATUS_STACK_OVERFLOW) instead of overrunning the array.
#pragma once
#include "cpt_device.cuh"
#include "cpt.h"

namespace cpt {

struct Hit { float t, u, v; uint32_t tri; };

__device__ __forceinline__ float slab_test(f3 o, f3 dinv, float ax, float ay, float az, float bx, float by, float bz)
{
    float tx0 = __fmul_rn(__fsub_rn(ax, o.x), dinv.x), tx1 = __fmul_rn(__fsub_rn(bx, o.x), dinv.x);
    float ty0 = __fmul_rn(__fsub_rn(ay, o.y), dinv.y), ty1 = __fmul_rn(__fsub_rn(by, o.y), dinv.y);
    float tz0 = __fmul_rn(__fsub_rn(az, o.z), dinv.z), tz1 = __fmul_rn(__fsub_rn(bz, o.z), dinv.z);
    float n = gmax(gmax(gmin(tx0, tx1), gmin(ty0, ty1)), gmin(tz0, tz1));
    float f = gmin(gmin(gmax(tx0, tx1), gmax(ty0, ty1)), gmax(tz0, tz1));
    return (n <= f && f > 0.0f) ? n : FLT_MAX;
}

__device__ __forceinline__ float tri_test(f3 o, f3 d, const float4* __restrict__ rec, float& u, float& v)
{
    float4 a = __ldg(rec), b = __ldg(rec + 1), c = __ldg(rec + 2);
    f3 p0 = mk3(a.x, a.y, a.z), e1 = mk3(b.x, b.y, b.z), e2 = mk3(c.x, c.y, c.z);
    f3 q = cross(d, e2);
    float det = dot(e1, q);
    if (det > -FLT_EPSILON && det < FLT_EPSILON) return FLT_MAX;
    float inv = __frcp_rn(det);
    f3 s = sub(o, p0);
    u = __fmul_rn(inv, dot(s, q));
    if (u < 0.f) return FLT_MAX;
    f3 r = cross(s, e1);
    v = __fmul_rn(inv, dot(d, r));
    if (v < 0.f || __fadd_rn(u, v) > 1.f) return FLT_MAX;
    float t = __fmul_rn(inv, dot(e2, r));
    return t >= 0.0f ? t : FLT_MAX;
}

// stack: this thread's column base in shared memory (s_stack + threadIdx.x).
template <bool kAny, int kBlock, bool kStats>
__device__ __forceinline__ Hit traverse(const float4* __restrict__ nodes, const float4* __restrict__ tris, f3 o, f3 d,
                                        uint32_t* stack, bool& overflow, uint32_t& n_nodes, uint32_t& n_tris)
{
    const f3 dinv = mk3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
    Hit best;
    best.t = FLT_MAX;
    best.u = 0.f;
    best.v = 0.f;
    best.tri = CPT_INVALID_INDEX;
    int sp = 0;
    uint32_t cur = 0;  // the root, Node::makeInternal(0)
    for (;;) {
        for (;;) {
            const float4* nd = nodes + 4 * (size_t)cur;
            const float4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2);
            const uint32_t word = __float_as_uint(__ldg(reinterpret_cast<const float*>(nd + 3)));
            if (kStats) ++n_nodes;
            const uint32_t li = word >> 2, ri = li + 1;
            const bool lint = word & 1u, rint = word & 2u;
            float lu = 0.f, lv = 0.f, ru = 0.f, rv = 0.f, hl, hr;
            if (lint) hl = slab_test(o, dinv, n0.x, n0.y, n0.z, n0.w, n1.x, n1.y);
            else { hl = tri_test(o, d, tris + 3 * (size_t)li, lu, lv); if (kStats) ++n_tris; }
            if (rint) hr = slab_test(o, dinv, n1.z, n1.w, n2.x, n2.y, n2.z, n2.w);
            else { hr = tri_test(o, d, tris + 3 * (size_t)ri, ru, rv); if (kStats) ++n_tris; }
            if (hl >= best.t && hr >= best.t) break;
            const bool sw = hr < hl;
            const float hc = sw ? hr : hl, hf = sw ? hl : hr;
            const uint32_t ic = sw ? ri : li, ifar = sw ? li : ri;
            const bool cint = sw ? rint : lint, fint = sw ? lint : rint;
            if (cint) {
                if (hf < best.t) {
                    if (fint) {
                        if (sp < CPT_TRAVERSAL_STACK) stack[(sp++) * kBlock] = ifar;
                        else overflow = true;
                    } else {
                        best.t = hf;
                        best.u = sw ? lu : ru;
                        best.v = sw ? lv : rv;
                        best.tri = ifar;
                        if (kAny) return best;
                    }
                }
                cur = ic;
            } else {
                best.t = hc;
                best.u = sw ? ru : lu;
                best.v = sw ? rv : lv;
                best.tri = ic;
                if (kAny) return best;
                break;
            }
        }
        if (sp == 0) break;
        cur = stack[(--sp) * kBlock];
    }
    return best;
}

}  // namespace cpt
