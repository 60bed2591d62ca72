// Closest-hit / any-hit traversal over the compact LBVH records and over the wide tree.
//
// Follows CUDA::trace (source/application/cuda/trace.h:73-169) decision for
// decision — both children tested (left first), both-farther-than-best pruning,
// nearer child first (ties to the left), the farther internal child pushed or
// the farther triangle recorded, a nearer triangle ending the descent — so the
// returned (t, triangle, u, v) are those of the reference, with the same
// Möller-Trumbore (intersection.h:28-59) and slab (intersection.h:106-117)
// arithmetic in round-to-nearest intrinsics.
//
// What changes is the memory side and the scheduling:
//  * one 96-B record per internal node (six 16-B loads, three 32-B sectors) holds
//    both children and the Node word. A child slot (10 words) is either the
//    child's box (internal child) or the child triangle itself — v0, the
//    triangle's index in the sorted array, v1 - v0, v2 - v0 (leaf child): the reference loads a 4-B Node, then a
//    24-B box or a 40-B triangle per child from separate arrays; here one round
//    trip fetches everything a visit needs. The stored edges are the same
//    subtractions the test performs, so the bits are unchanged.
//  * 1/d is computed once per ray instead of per box (same value).
//  * the node stack is CPT_TRAVERSAL_STACK deep like the reference's local array:
//    the first kSmemStack entries live in shared memory, one column per thread,
//    the rest (never reached on the test scenes) in local memory; a push beyond
//    the capacity is dropped and reported (CPT_STATUS_STACK_OVERFLOW) instead of
//    overrunning the array.
//  * traversal kernels are persistent: lanes take rays from a global pool, and a
//    warp takes new rays for its idle lanes once fewer than half of them still
//    trace, so a warp is not held by its slowest ray (per-ray node counts differ
//    by 100x on hairball scenes).
//
// The second half of the file traverses the compressed 8-wide tree (cpt_lbvh_wide)
// built over a binary tree: 80-B nodes with 8-bit child planes, the same triangle
// test on the binary leaf slot's words, triangle tests in warp batches and a refill
// once two lanes are idle.
#pragma once
#include <cuda_fp16.h>
#include "cpt_device.cuh"
#include "cpt.h"

namespace cpt {

constexpr int kSmemStack = 32;
#ifndef CPT_REFILL_LANES
#define CPT_REFILL_LANES 16
#endif
constexpr int kRefillLanes = CPT_REFILL_LANES;  // persistent traversal refills below this many busy lanes
constexpr int kNodeFloat4 = 6;  // 96-B node record
constexpr int kNodeFloats = 24;

struct Hit { float t, u, v; uint32_t tri; };

// Slab test with glm's select semantics (min(x,y) = x<y?x:y, max(x,y) = x>y?x:y).
// When every 1/d component is finite ("finite"), no product can be NaN, and then
// those selects and fminf/fmaxf return the same value (up to the sign of a zero,
// which no comparison below sees), so the single-instruction forms are used.
__device__ __forceinline__ float slab_test(f3 o, f3 dinv, bool finite, float ax, float ay, float az, float bx,
                                           float by, float bz)
{
    const float tx0 = __fmul_rn(__fsub_rn(ax, o.x), dinv.x), tx1 = __fmul_rn(__fsub_rn(bx, o.x), dinv.x);
    const float ty0 = __fmul_rn(__fsub_rn(ay, o.y), dinv.y), ty1 = __fmul_rn(__fsub_rn(by, o.y), dinv.y);
    const float tz0 = __fmul_rn(__fsub_rn(az, o.z), dinv.z), tz1 = __fmul_rn(__fsub_rn(bz, o.z), dinv.z);
    float n, f;
    if (finite) {
        n = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
        f = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    } else {
        n = gmax(gmax(gmin(tx0, tx1), gmin(ty0, ty1)), gmin(tz0, tz1));
        f = gmin(gmin(gmax(tx0, tx1), gmax(ty0, ty1)), gmax(tz0, tz1));
    }
    return (n <= f && f > 0.0f) ? n : FLT_MAX;
}

// Slab test for trees whose box distances only steer pruning (the split BVH):
// t = b * (1/d) - o * (1/d) in one fused multiply-add per plane. Valid when every
// 1/d component is finite (no inf * 0).
__device__ __forceinline__ float slab_test_fma(f3 odinv, f3 dinv, float ax, float ay, float az, float bx, float by,
                                               float bz)
{
    const float tx0 = fmaf(ax, dinv.x, -odinv.x), tx1 = fmaf(bx, dinv.x, -odinv.x);
    const float ty0 = fmaf(ay, dinv.y, -odinv.y), ty1 = fmaf(by, dinv.y, -odinv.y);
    const float tz0 = fmaf(az, dinv.z, -odinv.z), tz1 = fmaf(bz, dinv.z, -odinv.z);
    const float n = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fminf(tz0, tz1));
    const float f = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1));
    return (n <= f && f > 0.0f) ? n : FLT_MAX;
}

// Packed FP32 pairs (sm_100: add / sub / mul / fma .rn.f32x2). Each lane of the pair
// is rounded exactly as the scalar round-to-nearest operation on it, so a packed
// sequence gives the bits of the scalar one; it issues one instruction per pair.
// The wide tree's box test evaluates an axis's near and far plane with one packed
// fused multiply-add. The triangle test stays scalar: a packed Moller-Trumbore (the two
// cross products and the dot products that share a factor in pairs) gave a quarter of
// its cross-product lanes 1 ulp off the scalar sequence on the device (a packed
// multiply and subtract contracted into one fused operation), and exact hits are
// required here.
struct f2 { float x, y; };
__device__ __forceinline__ f2 mk2(float x, float y) { f2 r; r.x = x; r.y = y; return r; }
#define CPT_F2_OP(name, op)                                                                                    \
    __device__ __forceinline__ f2 name(f2 a, f2 b)                                                              \
    {                                                                                                         \
        f2 d;                                                                                                 \
        asm("{.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t" op            \
            " rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;}"                                                         \
            : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                  \
        return d;                                                                                             \
    }
CPT_F2_OP(add2, "add.rn.f32x2")
CPT_F2_OP(sub2, "sub.rn.f32x2")
CPT_F2_OP(mul2, "mul.rn.f32x2")
#undef CPT_F2_OP
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 d;
    asm("{.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\tmov.b64 rc, {%6, %7};\n\t"
        "fma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

// Möller-Trumbore on a slot (v0 = s[0..2], e1 = s[4..6], e2 = s[7..9]), without
// early exits: every lane of a warp runs the same instructions, and u, v, t are the
// values the reference computes; only the final predicate decides the hit.
// the two halves of w as floats (exact)
__device__ __forceinline__ f2 half_pair(uint32_t w)
{
    __half2 h;
    memcpy(&h, &w, 4);
    const float2 f = __half22float2(h);
    return mk2(f.x, f.y);
}

__device__ __forceinline__ float tri_test(f3 o, f3 d, const float* s, float& u, float& v)
{
    const f3 p0 = mk3(s[0], s[1], s[2]), e1 = mk3(s[4], s[5], s[6]), e2 = mk3(s[7], s[8], s[9]);
    const f3 q = cross(d, e2);
    const float det = dot(e1, q);
    const float inv = __frcp_rn(det);
    const f3 sv = sub(o, p0);
    u = __fmul_rn(inv, dot(sv, q));
    const f3 r = cross(sv, e1);
    v = __fmul_rn(inv, dot(d, r));
    const float t = __fmul_rn(inv, dot(e2, r));
    const bool hit = !(det > -FLT_EPSILON && det < FLT_EPSILON) && !(u < 0.f) && !(v < 0.f) &&
                     !(__fadd_rn(u, v) > 1.f) && t >= 0.0f;
    return hit ? t : FLT_MAX;
}

// Per-ray traversal state.
struct TraceState {
    const float4* nodes;  // the node array of the ray's BVH
    uint32_t max_visits;  // node fetches allowed (a valid tree needs at most its n - 1 internal nodes)
    f3 o, d, dinv;
    bool finite;  // all components of 1/d finite
    Hit best;
    uint32_t cur;
    int sp;
    uint32_t visits;  // node fetches
    uint32_t tests;   // triangle tests
    bool fast;        // fused slab test (split BVH and finite 1/d)
    f3 odinv;         // o * (1/d), for the fused slab test
};

// Visit bound word: bit 31 set = a tree whose box distances only steer pruning
// (the split BVH), which may use the fused slab test.
constexpr uint32_t kFastSlabBit = 0x80000000u;

__device__ __forceinline__ void trace_init(TraceState& s, const float4* nodes, uint32_t max_visits, f3 o, f3 d)
{
    s.nodes = nodes;
    s.max_visits = max_visits & ~kFastSlabBit;
    s.o = o;
    s.d = d;
    s.dinv = mk3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
    s.finite = isfinite(s.dinv.x) && isfinite(s.dinv.y) && isfinite(s.dinv.z);
    s.fast = (max_visits & kFastSlabBit) && s.finite;
    s.odinv = mk3(o.x * s.dinv.x, o.y * s.dinv.y, o.z * s.dinv.z);
    s.best.t = FLT_MAX;
    s.best.u = 0.f;
    s.best.v = 0.f;
    s.best.tri = CPT_INVALID_INDEX;
    s.cur = 0;  // the root, Node::makeInternal(0)
    s.sp = 0;
    s.visits = 0;
    s.tests = 0;
}

template <int kBlock>
__device__ __forceinline__ void stack_push(uint32_t* smem_col, uint32_t* spill, int& sp, uint32_t v, bool& overflow)
{
    if (sp < kSmemStack) smem_col[sp * kBlock] = v;
    else if (sp < CPT_TRAVERSAL_STACK) spill[sp - kSmemStack] = v;
    else { overflow = true; return; }
    ++sp;
}

template <int kBlock>
__device__ __forceinline__ uint32_t stack_pop(const uint32_t* smem_col, const uint32_t* spill, int& sp)
{
    --sp;
    return sp < kSmemStack ? smem_col[sp * kBlock] : spill[sp - kSmemStack];
}

// One node visit of trace.h:104-165. Returns true when the ray is finished
// (stack empty after a pop, or — any-hit — a triangle was recorded).
template <bool kAny, int kBlock, bool kStats>
__device__ __forceinline__ bool trace_step(TraceState& s, uint32_t* smem_col, uint32_t* spill, bool& overflow,
                                           uint32_t& n_nodes, uint32_t& n_tris)
{
    if (++s.visits > s.max_visits) { overflow = true; return true; }
    const float4* nd = s.nodes + kNodeFloat4 * (size_t)s.cur;
    float w[kNodeFloats];
#pragma unroll
    for (int k = 0; k < kNodeFloat4; ++k) {
        const float4 f = __ldg(nd + k);
        w[4 * k] = f.x; w[4 * k + 1] = f.y; w[4 * k + 2] = f.z; w[4 * k + 3] = f.w;
    }
    const uint32_t word = __float_as_uint(w[20]);
    if (kStats) ++n_nodes;
    const uint32_t li = word >> 2, ri = __float_as_uint(w[21]);
    const bool lint = word & 1u, rint = word & 2u;
    // the triangle a leaf child stands for: its slot's index word (the leaf position
    // in an LBVH over the triangles, the piece's triangle in a split BVH)
    const uint32_t tl = __float_as_uint(w[3]), tr = __float_as_uint(w[13]);
    if (kStats) {
        const uint32_t t = (lint ? 0u : 1u) + (rint ? 0u : 1u);
        n_tris += t;
        s.tests += t;
    }
    float lu = 0.f, lv = 0.f, ru = 0.f, rv = 0.f;
    // Both slab tests run on every lane (a leaf slot's result is discarded), then
    // one Möller-Trumbore code path serves the first leaf child, left or right,
    // and a second one only lanes whose two children are both leaves.
    float hl, hr;
    if (s.fast) {
        hl = slab_test_fma(s.odinv, s.dinv, w[0], w[1], w[2], w[3], w[4], w[5]);
        hr = slab_test_fma(s.odinv, s.dinv, w[10], w[11], w[12], w[13], w[14], w[15]);
    } else {
        hl = slab_test(s.o, s.dinv, s.finite, w[0], w[1], w[2], w[3], w[4], w[5]);
        hr = slab_test(s.o, s.dinv, s.finite, w[10], w[11], w[12], w[13], w[14], w[15]);
    }
    if (!lint || !rint) {
        float t0[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) t0[k] = lint ? w[10 + k] : w[k];
        float u0, v0;
        const float h0 = tri_test(s.o, s.d, t0, u0, v0);
        if (!lint) { hl = h0; lu = u0; lv = v0; }
        else { hr = h0; ru = u0; rv = v0; }
        if (!lint && !rint) hr = tri_test(s.o, s.d, w + 10, ru, rv);
    }
    bool pop = false;
    if (hl >= s.best.t && hr >= s.best.t) {
        pop = true;
    } else {
        const bool sw = hr < hl;
        const float hc = sw ? hr : hl, hf = sw ? hl : hr;
        const uint32_t ic = sw ? ri : li, ifar = sw ? li : ri;
        const bool cint = sw ? rint : lint, fint = sw ? lint : rint;
        if (cint) {
            if (hf < s.best.t) {
                if (fint) {
                    stack_push<kBlock>(smem_col, spill, s.sp, ifar, overflow);
                } else {
                    s.best.t = hf;
                    s.best.u = sw ? lu : ru;
                    s.best.v = sw ? lv : rv;
                    s.best.tri = sw ? tl : tr;
                    if (kAny) return true;
                }
            }
            s.cur = ic;
        } else {
            s.best.t = hc;
            s.best.u = sw ? ru : lu;
            s.best.v = sw ? rv : lv;
            s.best.tri = sw ? tr : tl;
            if (kAny) return true;
            pop = true;
        }
    }
    if (pop) {
        if (s.sp == 0) return true;
        s.cur = stack_pop<kBlock>(smem_col, spill, s.sp);
    }
    return false;
}

// Whole traversal of one ray by one thread (shadow rays inside the shade kernel).
template <bool kAny, int kBlock>
__device__ __forceinline__ Hit traverse(const float4* __restrict__ nodes, f3 o, f3 d, uint32_t* smem_col, bool& overflow,
                                        uint32_t max_visits)
{
    TraceState s;
    trace_init(s, nodes, max_visits, o, d);
    uint32_t spill[CPT_TRAVERSAL_STACK - kSmemStack];
    uint32_t nn = 0, nt = 0;
    while (!trace_step<kAny, kBlock, false>(s, smem_col, spill, overflow, nn, nt)) {
    }
    return s.best;
}

// ---------------------------------------------------------------------------
// Compressed 8-wide BVH (cpt_lbvh_wide). A wide node is five float4 (child box planes
// p + q * 2^e, q one byte):
//   n0 = (p.x, p.y, p.z, bits of 2^e_z >> 16 | internal slot mask << 24)
//   n1 = (first internal child, first triangle record,
//         leaf slot mask | slots with 2+ records << 8 | slots with 3 records << 16,
//         bits of 2^e_x >> 16 | bits of 2^e_y & 0xFFFF0000)
//   n2, n3, n4 = the planes of x, y, z: word j holds slots 2j, 2j+1 as bytes (lo, hi, lo, hi)
// A leaf slot holds 1 to 3 triangle records (a binary subtree of up to three leaves under
// one box). Record j of the leaf slot of rank r among the node's L leaf slots is the
// node's record j * L + r (layers of L records; a slot with fewer records leaves holes).
// The ray carries a node group — the hit internal slots of one node still to visit, in
// the order k ^ octant(ray) — and up to three triangle groups — the records of the hit
// leaf slots of nodes visited, in visiting order: bits 8j + s for record j of slot s, the
// node's leaf slot mask in bits 24-31. A
// step tests one triangle of the first triangle group and, unless every group slot is
// taken, visits the next node of the node group (the rest of the group goes on the
// stack; the node's triangle group queues behind), or pops a group. The triangle test
// is tri_test on the binary leaf slot's words, so a hit's t, u, v are unchanged.
constexpr int kWideSmemStack = 16;  // stack entries (2 words) per thread in shared memory
constexpr float kWideGrow = 1.0f + 1.0f / 262144.0f;  // relative slack of a wide child's box test
// Records a leaf slot holds at most: binary subtrees of up to this many leaves become one
// leaf slot of their parent wide node instead of a wide node of their own; a wide tree
// over L binary leaves has kWideRecordLayers * L record positions. C2: 544.5 Mrays/s
// with 1 (65.9 node visits and 20.1 triangle tests per ray), 559.8 with 2 (63.7, 20.9),
// 559.6 with 3 (61.7, 23.7).
#ifndef CPT_WIDE_LEAF_MAX
#define CPT_WIDE_LEAF_MAX 2
#endif
constexpr uint32_t kWideRecordLayers = CPT_WIDE_LEAF_MAX;
static_assert(kWideRecordLayers >= 1 && kWideRecordLayers <= 3, "a leaf slot holds 1 to 3 records");
constexpr uint32_t kWideRecBits = 0x00FFFFFFu;  // a triangle group's record bits
// The wide traversal refills once two lanes of the warp are idle (fewer than 31 busy):
// its steps are long (8 child boxes), so idle lanes cost more than the refill's ballot
// and atomic (C2 with one triangle test per step: 313 Mrays/s at 32, 302 at 28, 283 at
// 24, 242 at 16, 196 at 8; with the tests batched per warp: 505.5 / 506.0 at 32,
// 514.7 / 514.3 at 31, 513.6 / 513.6 at 30, 509.0 at 29, 506.2 at 28).
#ifndef CPT_WIDE_REFILL_LANES
#define CPT_WIDE_REFILL_LANES 31
#endif
constexpr int kWideRefillLanes = CPT_WIDE_REFILL_LANES;
// A lane with triangles still to test may visit its next node in the same step, the
// node's triangle group queuing behind the first (up to three groups pending): steps
// that were a triangle test for some lanes and a node visit for the others become both
// for most lanes (C2: 370 Mrays/s with one group, 413 with two, 420 with three).
constexpr float kWideFarInv = 1099511627776.0f;  // 2^40: 1/d of a zero direction component
// Triangle tests in warp batches: a lane's pending triangles wait (it keeps visiting
// nodes, its groups queue up) until at least this many lanes of the warp have some, or
// one lane must test (all three group slots taken, or no node left to visit), so the
// test runs with more lanes at once (C2, lanes that test per test step 9.2 of 32 without
// it; threshold 8 / 12 / 16 / 20 / 24: 491.9 / 502.6 / 507.2 / 505.6 / 506.4 Mrays/s
// against 493.9; 0 turns it off). Every step still consumes a node, a stack entry or a
// triangle of every live lane, or ends its ray.
#ifndef CPT_WIDE_TRI_BATCH
#define CPT_WIDE_TRI_BATCH 16
#endif
constexpr int kWideTriBatch = CPT_WIDE_TRI_BATCH;

struct WideState {
    const float4* nodes;
    const float4* tris;
    uint32_t max_visits;  // wide node fetches allowed (the wide tree's node capacity)
    uint32_t tri_cap;     // triangle records
    f3 o, d, dinv;
    uint32_t oct;         // direction sign bits (x: 1, y: 2, z: 4)
    Hit best;
    uint32_t cbase, gbits;  // node group: first child; bits 0-7 hit slots in visit order, 8-15 internal mask
    uint32_t tbase, tbits;  // triangle group: first record; records to test (kWideRecBits), leaf mask << 24
    uint32_t tbase2, tbits2;  // a second triangle group, queued behind the first
    uint32_t tbase3, tbits3;  // and a third
    int sp;
    uint32_t visits, tests;
};

__device__ __forceinline__ void wide_init(WideState& s, const float4* nodes, const float4* tris, uint32_t max_visits,
                                          f3 o, f3 d)
{
    s.nodes = nodes;
    s.tris = tris;
    s.max_visits = max_visits;
    s.tri_cap = kWideRecordLayers * (max_visits + 1);
    s.o = o;
    s.d = d;
    const float ix = __frcp_rn(d.x), iy = __frcp_rn(d.y), iz = __frcp_rn(d.z);
    s.dinv = mk3(isfinite(ix) ? ix : copysignf(kWideFarInv, d.x), isfinite(iy) ? iy : copysignf(kWideFarInv, d.y),
                 isfinite(iz) ? iz : copysignf(kWideFarInv, d.z));
    s.oct = (s.dinv.x < 0.f ? 1u : 0u) | (s.dinv.y < 0.f ? 2u : 0u) | (s.dinv.z < 0.f ? 4u : 0u);

    s.best.t = FLT_MAX;
    s.best.u = 0.f;
    s.best.v = 0.f;
    s.best.tri = CPT_INVALID_INDEX;
    s.cbase = 0;  // the root, wide node 0: the one internal slot (0) of a virtual parent, visited first
    s.gbits = (1u << s.oct) | (1u << 8);
    s.tbase = 0;
    s.tbits = 0;
    s.tbase2 = 0;
    s.tbits2 = 0;
    s.tbase3 = 0;
    s.tbits3 = 0;
    s.sp = 0;
    s.visits = 0;
    s.tests = 0;
}

__device__ __forceinline__ float fmax3(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

__device__ __forceinline__ float fmin3(float a, float b, float c)
{
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// bit k of the result = bit (k ^ oct) of x (8-bit masks)
__device__ __forceinline__ uint32_t xor_permute8(uint32_t x, uint32_t oct)
{
    x = (oct & 1u) ? (((x & 0x55u) << 1) | ((x >> 1) & 0x55u)) : x;
    x = (oct & 2u) ? (((x & 0x33u) << 2) | ((x >> 2) & 0x33u)) : x;
    x = (oct & 4u) ? (((x & 0x0Fu) << 4) | ((x >> 4) & 0x0Fu)) : x;
    return x;
}

// Fills the block's octant permutation table (byte oct * 256 + x = xor_permute8(x, oct));
// every thread of the block calls it, before any traversal.
__device__ __forceinline__ void wide_perm_table(uint8_t* perm)
{
    for (uint32_t i = threadIdx.x; i < 2048u; i += blockDim.x) perm[i] = (uint8_t)xor_permute8(i & 255u, i >> 8);
    __syncthreads();
}

template <int kBlock>
__device__ __forceinline__ void wide_push(uint2* smem_col, uint2* spill, int& sp, uint2 v, bool& overflow)
{
    if (sp < kWideSmemStack) smem_col[sp * kBlock] = v;
    else if (sp < CPT_TRAVERSAL_STACK) spill[sp - kWideSmemStack] = v;
    else { overflow = true; return; }
    ++sp;
}

template <int kBlock>
__device__ __forceinline__ uint2 wide_pop(const uint2* smem_col, const uint2* spill, int& sp)
{
    --sp;
    return sp < kWideSmemStack ? smem_col[sp * kBlock] : spill[sp - kWideSmemStack];
}

// The children of a wide node (five float4 n0..n4) whose boxes the ray's interval
// [0, best] meets: bit i for slot i.
__device__ __forceinline__ uint32_t wide_child_hits(const WideState& s, float4 n0, float4 n1, float4 n2, float4 n3,
                                                    float4 n4)
{
    // per-axis scales 2^e: the float bits e << 23 are stored as half-words (x, y in n1.w,
    // z in the low half of n0.w), moved to the high half by one byte permute each
    const uint32_t h01 = __float_as_uint(n1.w), h2 = __float_as_uint(n0.w);
    const float sx = __uint_as_float(__byte_perm(h01, 0u, 0x1044u)), sy = __uint_as_float(h01 & 0xFFFF0000u),
                sz = __uint_as_float(__byte_perm(h2, 0u, 0x1044u));
    // plane t = q * (2^e / d) + (p - o) / d, evaluated as (1024 + q) * a + (b - 1024 * a):
    // the folded offset rounds at the scale of b, well inside the build's spare quantum
    const float adx = sx * s.dinv.x, ady = sy * s.dinv.y, adz = sz * s.dinv.z;
    const f2 ax2 = mk2(adx, adx), ay2 = mk2(ady, ady), az2 = mk2(adz, adz);
    const float bdx = fmaf(-1024.0f, adx, (n0.x - s.o.x) * s.dinv.x);
    const float bdy = fmaf(-1024.0f, ady, (n0.y - s.o.y) * s.dinv.y);
    const float bdz = fmaf(-1024.0f, adz, (n0.z - s.o.z) * s.dinv.z);
    const f2 bx2 = mk2(bdx, bdx), by2 = mk2(bdy, bdy), bz2 = mk2(bdz, bdz);
    const uint32_t px[4] = {__float_as_uint(n2.x), __float_as_uint(n2.y), __float_as_uint(n2.z), __float_as_uint(n2.w)};
    const uint32_t py[4] = {__float_as_uint(n3.x), __float_as_uint(n3.y), __float_as_uint(n3.z), __float_as_uint(n3.w)};
    const uint32_t pz[4] = {__float_as_uint(n4.x), __float_as_uint(n4.y), __float_as_uint(n4.z), __float_as_uint(n4.w)};
    // byte permute selectors: result bytes (near plane, 0x64, far plane, 0x64) of (word,
    // 0x64646464) are the halves 1024 + q_near, 1024 + q_far; the near plane is hi for a
    // negative direction; odd slots read bytes 2, 3
    uint32_t oct = s.oct;
    asm volatile("" : "+r"(oct));  // derived per node: loop-invariant copies would cost registers
    const uint32_t px0 = (oct & 1u) ? 0x4041u : 0x4140u, py0 = (oct & 2u) ? 0x4041u : 0x4140u,
                   pz0 = (oct & 4u) ? 0x4041u : 0x4140u;
    const uint32_t sel[2][3] = {{px0, py0, pz0}, {px0 + 0x0202u, py0 + 0x0202u, pz0 + 0x0202u}};
    const float tlim = s.best.t;
    uint32_t hm = 0;
#pragma unroll
    for (int i = 0; i < 8; i += 2) {  // two children at a time
        float tn[2], tf[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            // one packed fused multiply-add per axis gives (t_near, t_far), each lane
            // rounded as the scalar fmaf
            const f2 tx = fma2(half_pair(__byte_perm(px[i >> 1], 0x64646464u, sel[k][0])), ax2, bx2);
            const f2 ty = fma2(half_pair(__byte_perm(py[i >> 1], 0x64646464u, sel[k][1])), ay2, by2);
            const f2 tz = fma2(half_pair(__byte_perm(pz[i >> 1], 0x64646464u, sel[k][2])), az2, bz2);
            tn[k] = fmaxf(fmax3(tx.x, ty.x, tz.x), 0.0f);
            tf[k] = fminf(fmin3(tx.y, ty.y, tz.y), tlim);
        }
        // [max(tn, 0), min(tf, best) * (1 + 2^-18)] non-empty: the far end grows by a
        // relative 2^-18, which covers the rounding of (p - o) / d for ray origins at any
        // distance; both children in one packed multiply
        const f2 g = mul2(mk2(tf[0], tf[1]), mk2(kWideGrow, kWideGrow));
        hm |= (tn[0] <= g.x ? 1u : 0u) << i;
        hm |= (tn[1] <= g.y ? 1u : 0u) << (i + 1);
    }
    return hm;
}

// One step; returns true when the ray is finished.
// perm: xor_permute8 as a table in shared memory, byte oct * 256 + x (wide_perm_table).
template <bool kAny, int kBlock, bool kStats>
__device__ __forceinline__ bool wide_step(WideState& s, uint2* smem_col, uint2* spill, bool& overflow,
                                          uint32_t& n_nodes, uint32_t& n_tris, const uint8_t* perm,
                                          bool test_tri = true)
{
    if (test_tri && (s.tbits & kWideRecBits)) {
        // the lowest record bit, 8j + slot (the leaf mask lies above): record j * L + rank
        // of the slot = the set bits below it in the leaf mask copied into bytes 0-2
        const uint32_t t1 = s.tbits - 1u;
        const uint32_t below = (s.tbits ^ t1) >> 1;
        const uint32_t idx = s.tbase + __popc(((s.tbits >> 24) * 0x010101u) & below);
        s.tbits &= t1;
        if (idx >= s.tri_cap) { overflow = true; return true; }
        const float4 a = __ldg(s.tris + 3 * (size_t)idx), b = __ldg(s.tris + 3 * (size_t)idx + 1),
                     c = __ldg(s.tris + 3 * (size_t)idx + 2);
        const float w[10] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, c.x, c.y, c.z};
        float u, v;
        const float t = tri_test(s.o, s.d, w, u, v);
        if (kStats) { ++n_tris; ++s.tests; }
        if (t < s.best.t) {
            s.best.t = t;
            s.best.u = u;
            s.best.v = v;
            s.best.tri = __float_as_uint(a.w);
            if (kAny) return true;
        }
        if (!(s.tbits & kWideRecBits) && (s.tbits2 & kWideRecBits)) {  // the queued groups move up
            s.tbase = s.tbase2;
            s.tbits = s.tbits2;
            s.tbase2 = s.tbase3;
            s.tbits2 = s.tbits3;
            s.tbits3 = 0;
        }
        if (s.tbits3 & kWideRecBits) return false;  // every group slot pending: no node visit this step
    }
    if (!(s.gbits & 0xFFu)) {
        if (s.sp == 0) return !(s.tbits & kWideRecBits);  // done once the last triangles are tested
        const uint2 g = wide_pop<kBlock>(smem_col, spill, s.sp);
        s.cbase = g.x;
        s.gbits = g.y;
    }
    const uint32_t k = __ffs(s.gbits & 0xFFu) - 1;
    s.gbits &= ~(1u << k);
    const uint32_t slot = k ^ s.oct;
    const uint32_t child = s.cbase + __popc((s.gbits >> 8) & ((1u << slot) - 1u));
    if (s.gbits & 0xFFu) wide_push<kBlock>(smem_col, spill, s.sp, make_uint2(s.cbase, s.gbits), overflow);
    if (++s.visits > s.max_visits || child >= s.max_visits) { overflow = true; return true; }
    if (kStats) ++n_nodes;
    const float4* nd = s.nodes + 5 * (size_t)child;
    const float4 n0 = __ldg(nd), n1 = __ldg(nd + 1), n2 = __ldg(nd + 2), n3 = __ldg(nd + 3), n4 = __ldg(nd + 4);
    const uint32_t imask = __float_as_uint(n0.w) >> 24, lw = __float_as_uint(n1.z);
    const uint32_t hm = wide_child_hits(s, n0, n1, n2, n3, n4);
    s.cbase = __float_as_uint(n1.x);
    s.gbits = (uint32_t)perm[(s.oct << 8) | (hm & imask)] | (imask << 8);
    // the hit slots' records: the hit mask copied into bytes 0-2, masked by the slots
    // holding a first / second / third record; the leaf mask above
    const uint32_t recs = ((hm * 0x010101u) & lw) | (lw << 24);
    if (s.tbits & kWideRecBits) {  // triangles still pending: the new group queues behind them
        if (s.tbits2 & kWideRecBits) {
            s.tbase3 = __float_as_uint(n1.y);
            s.tbits3 = recs;
            return false;
        }
        s.tbase2 = __float_as_uint(n1.y);
        s.tbits2 = recs;
        return false;
    }
    s.tbase = __float_as_uint(n1.y);
    s.tbits = recs;
    return false;
}

// Persistent traversal of `n` rays: ray i is (origin, direction) = rays[2i], rays[2i+1].
// nodes_of(w, max_visits) returns the node array (and the visit bound) for the word
// w carried in the direction's .w (a view index, or unused). kTmax: the origin's .w
// is the ray's far limit (a triangle at t >= it is not a hit; shadow rays toward a
// point); otherwise the ray is unbounded. done(i, state) is called once per ray when
// its traversal ends. Idle lanes take rays from *pool in warp-sized grabs (one
// atomic per warp) whenever fewer than kRefillLanes lanes of the warp still trace
// (at most kSteps node visits apart): refilling at every finished ray costs more in
// bookkeeping than the idle lanes do (C2: 16 lanes, 228 vs 194 Mrays/s).
// order (nullable): rays are taken in the order order[0], order[1], ... (a
// permutation of 0..n-1); done() still receives the ray's own index.
template <bool kAny, int kBlock, bool kStats, int kSteps, bool kTmax, typename NodesOf, typename Done>
__device__ __forceinline__ void persistent_trace(NodesOf nodes_of, const float4* __restrict__ rays, uint32_t n,
                                                 uint32_t* __restrict__ pool, uint32_t* smem_col, bool& overflow,
                                                 uint32_t& n_nodes, uint32_t& n_tris, const uint32_t* __restrict__ order,
                                                 Done done, uint32_t refill = 0)
{
    const uint32_t refill_below = refill ? refill : (uint32_t)kRefillLanes;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t spill[CPT_TRAVERSAL_STACK - kSmemStack];
    TraceState s;
    uint32_t ray = CPT_INVALID_INDEX;
    bool drained = false;
    for (;;) {
        if (!drained) {
            const bool idle = ray == CPT_INVALID_INDEX;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, idle);
            if (m) {
                const int leader = __ffs(m) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(pool, (uint32_t)__popc(m));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (base + (uint32_t)__popc(m) >= n) drained = true;
                if (idle) {
                    const uint32_t r = base + (uint32_t)__popc(m & lt_mask);
                    if (r < n) {
                        ray = order ? order[r] : r;
                        if (ray < n) {
                            const float4 ro = rays[2 * (size_t)ray], rd = rays[2 * (size_t)ray + 1];
                            uint32_t mv;
                            const float4* nodes = nodes_of(__float_as_uint(rd.w), mv);
                            trace_init(s, nodes, mv, mk3(ro.x, ro.y, ro.z), mk3(rd.x, rd.y, rd.z));
                            if (kTmax) s.best.t = ro.w;
                        } else {  // a ray order left void by a failed sort
                            overflow = true;
                            ray = CPT_INVALID_INDEX;
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, ray != CPT_INVALID_INDEX) == 0) break;
        // Step every lane that holds a ray; go back for more rays once fewer than
        // kRefillLanes lanes are busy (or after kSteps steps), unless the pool is empty.
#pragma unroll 1
        for (int k = 1;; ++k) {
            if (ray != CPT_INVALID_INDEX &&
                trace_step<kAny, kBlock, kStats>(s, smem_col, spill, overflow, n_nodes, n_tris)) {
                done(ray, s);
                ray = CPT_INVALID_INDEX;
            }
            const unsigned live = __ballot_sync(0xFFFFFFFFu, ray != CPT_INVALID_INDEX);
            if (live == 0) break;
            if (!drained && ((uint32_t)__popc(live) < refill_below || k >= kSteps)) break;
        }
    }
}

// persistent_trace over wide BVHs: wide_of(w, max_visits, tris) returns the wide
// node array, its node capacity and its triangle records for the word w of the
// direction's .w. Same refill rule and far-limit convention as persistent_trace.
template <bool kAny, int kBlock, bool kStats, int kSteps, bool kTmax, typename WideOf, typename Done>
__device__ __forceinline__ void persistent_trace_wide(WideOf wide_of, const float4* __restrict__ rays, uint32_t n,
                                                      uint32_t* __restrict__ pool, uint2* smem_col, bool& overflow,
                                                      uint32_t& n_nodes, uint32_t& n_tris,
                                                      const uint32_t* __restrict__ order, Done done,
                                                      uint32_t refill = 0)
{
    const uint32_t refill_below = refill ? refill : (uint32_t)kWideRefillLanes;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    __shared__ uint8_t s_perm[2048];
    wide_perm_table(s_perm);
    uint2 spill[CPT_TRAVERSAL_STACK - kWideSmemStack];
    WideState s;
    uint32_t ray = CPT_INVALID_INDEX;
    bool drained = false;
    for (;;) {
        if (!drained) {
            const bool idle = ray == CPT_INVALID_INDEX;
            const unsigned m = __ballot_sync(0xFFFFFFFFu, idle);
            if (m) {
                const int leader = __ffs(m) - 1;
                uint32_t base = 0;
                if ((int)lane == leader) base = atomicAdd(pool, (uint32_t)__popc(m));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (base + (uint32_t)__popc(m) >= n) drained = true;
                if (idle) {
                    const uint32_t r = base + (uint32_t)__popc(m & lt_mask);
                    if (r < n) {
                        ray = order ? order[r] : r;
                        if (ray < n) {
                            const float4 ro = rays[2 * (size_t)ray], rd = rays[2 * (size_t)ray + 1];
                            uint32_t mv;
                            const float4* tris;
                            const float4* nodes = wide_of(__float_as_uint(rd.w), mv, tris);
                            wide_init(s, nodes, tris, mv, mk3(ro.x, ro.y, ro.z), mk3(rd.x, rd.y, rd.z));
                            if (kTmax) s.best.t = ro.w;
                        } else {  // a ray order left void by a failed sort
                            overflow = true;
                            ray = CPT_INVALID_INDEX;
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, ray != CPT_INVALID_INDEX) == 0) break;
#pragma unroll 1
        for (int k = 1;; ++k) {
            bool test_tri = true;
            if (kWideTriBatch) {
                // the warp tests triangles when enough lanes have some pending, or when a lane
                // must (every group slot taken, or no node left to visit)
                const bool live = ray != CPT_INVALID_INDEX;
                const bool want = live && (s.tbits & kWideRecBits);
                const bool must = want && ((s.tbits3 & kWideRecBits) || (!(s.gbits & 0xFFu) && s.sp == 0));
                const unsigned bw = __ballot_sync(0xFFFFFFFFu, want);
                test_tri = __ballot_sync(0xFFFFFFFFu, must) != 0u || __popc(bw) >= kWideTriBatch;
            }
            if (ray != CPT_INVALID_INDEX &&
                wide_step<kAny, kBlock, kStats>(s, smem_col, spill, overflow, n_nodes, n_tris, s_perm, test_tri)) {
                done(ray, s);
                ray = CPT_INVALID_INDEX;
            }
            const unsigned live = __ballot_sync(0xFFFFFFFFu, ray != CPT_INVALID_INDEX);
            if (live == 0) break;
            if (!drained && ((uint32_t)__popc(live) < refill_below || k >= kSteps)) break;
        }
    }
}

// persistent_trace of unbounded rays whose hit goes to hits[i] = (t, u, v, triangle).
// ray_stats (nullable, with kStats): per ray (node fetches, triangle tests).
template <bool kAny, int kBlock, bool kStats, int kSteps, typename NodesOf>
__device__ __forceinline__ void persistent_trace_views(NodesOf nodes_of, const float4* __restrict__ rays, uint32_t n,
                                                       float4* __restrict__ hits, uint32_t* __restrict__ pool,
                                                       uint32_t* smem_col, bool& overflow, uint32_t& n_nodes,
                                                       uint32_t& n_tris, const uint32_t* __restrict__ order,
                                                       uint2* __restrict__ ray_stats = nullptr, uint32_t refill = 0)
{
    persistent_trace<kAny, kBlock, kStats, kSteps, false>(
        nodes_of, rays, n, pool, smem_col, overflow, n_nodes, n_tris, order,
        [&](uint32_t ray, const TraceState& s) {
            hits[ray] = make_float4(s.best.t, s.best.u, s.best.v, __uint_as_float(s.best.tri));
            if (kStats && ray_stats) ray_stats[ray] = make_uint2(s.visits, s.tests);
        },
        refill);
}

}  // namespace cpt
