// Compressed 8-wide traversal BVH (cpt_lbvh_wide): an extension with no reference
// counterpart, built from the binary traversal tree in use (the split tree when one
// was built, else the LBVH's nodes). Hits are those of the binary tree up to the order
// in which exactly equal distances are found: every triangle keeps its arithmetic
// (the leaf record holds the binary leaf slot's words), only the culling boxes change.
//
// Collapse: top-down, level by level of the wide tree inside one cooperative launch
// (k_wide_levels). A wide node starts from
// its binary node's two children and repeatedly opens the internal child of largest
// surface area until it has 8 children or only leaves. Its children go to slots by
// direction (Ylitie, Karras, Laine, "Efficient Incoherent Ray Traversal on GPUs
// Through Compressed Wide BVHs", HPG 2017): slot s is meant to be met first by rays
// whose direction has sign pattern s, so that visiting the slots in the order
// k ^ octant(ray), k = 0..7, is near-to-far; children are assigned greedily by the
// smallest projection of their centre on the octant's diagonal. After the collapse, an
// internal child whose binary subtree has up to kWideRecordLayers (2) leaves becomes a
// leaf slot holding those triangles (one box for them, no wide node of its own: C2's
// 8-wide tree had 5.2 M two-leaf and 2.0 M three-leaf nodes among 14.0 M). Internal children are allocated
// consecutively (one atomic per node) and queued for the next level; the leaf slots'
// triangle records likewise, in layers (record j of the leaf slot of rank r among L at
// j * L + r).
//
// Quantization: the node box, widened by a margin m, gives a per-axis power-of-two
// scale 2^e with (hi - lo + 2m) <= 253 * 2^e and the origin p = lo - m - 2^e (rounded
// down); a child box, widened by the same m, is stored as qlo = floor((lo - m - p) /
// 2^e) - 1, qhi = ceil((hi + m - p) / 2^e) + 1. The traversal evaluates a plane as
// fma(1024 + q, 2^e / d, (p - o) / d - 1024 * 2^e / d) (the byte read as the half
// 1024 + q, a slot's lo and hi bytes side by side), whose folded offset errs by far less
// than half a quantum (the spare quantum on each side covers it); m = 2^-20 x
// (largest root-box coordinate magnitude + root-box diagonal) covers the rounding of
// the quantized planes at the scene's scale, and the traversal's relative slack of
// 2^-18 on the far end of each interval covers the rounding of (p - o) / d, which
// grows with the distance of the ray origin.
// A leaf child's box is its triangle's box intersected with its binary parent's box
// (the binary parent of a split piece is bounded by the pieces, the triangle is not).
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"
#include "lbvh_common.cuh"
#include "traverse.cuh"
#include <cooperative_groups.h>

namespace cpt {
namespace {

constexpr int kWideBlock = 128;
constexpr int kWideLevels = 96;
constexpr uint32_t kLeafRef = 0x80000000u;
constexpr int kCtrWords = 4 + kWideLevels + 2;  // alloc nodes, alloc tris, done blocks, margin | level bounds

// Surface-area collapse (flag CPT_WIDE_SAH): which binary nodes become a wide node's children is
// chosen by the cost of each subtree as at most i children of a wide node, i = 1..8,
// computed bottom-up over the binary tree (Ylitie, Karras and Laine, "Efficient
// Incoherent Ray Traversal on GPUs Through Compressed Wide BVHs", HPG 2017, section
// 3.1, restated): for node n with children a, b and box area A,
//   D(n, j) = min over k in 1..j-1 of C(a, k) + C(b, j - k)
//   C(n, 1) = min(A * kSahNode + D(n, 8),                       n a wide node
//                 A * kSahPrim * P(n) if P(n) <= kWideRecordLayers)  n one leaf slot
//   C(n, j) = min(D(n, j), C(n, j - 1)) for j >= 2
// with a binary leaf costing its (clipped) box area times kSahPrim for every j, and
// P(n) the leaves under n. Without the flag the collapse opens the internal child of
// largest area until the node has 8 children.
#ifndef CPT_WIDE_SAH_PRIM
#define CPT_WIDE_SAH_PRIM 0.3f
#endif
constexpr float kSahNode = 1.0f, kSahPrim = CPT_WIDE_SAH_PRIM;
// choice word of a binary internal node: bit 0 one leaf slot; bit j - 1 (j = 2..8): C(n, j)
// = C(n, j - 1); bits 8 + 3 (j - 2): the k of D(n, j); bits 29-31: P(n), 7 meaning 7 or more
__device__ __forceinline__ bool sah_leaf(uint32_t c) { return c & 1u; }
__device__ __forceinline__ bool sah_reduce(uint32_t c, int j) { return (c >> (j - 1)) & 1u; }
__device__ __forceinline__ int sah_split(uint32_t c, int j) { return (int)((c >> (8 + 3 * (j - 2))) & 7u); }
__device__ __forceinline__ uint32_t sah_leaves(uint32_t c) { return c >> 29; }

struct WideScratch {
    float4* queue;  // per wide node: (box lo, binary node) (box hi, 0)
    uint32_t* ctr;
    uint32_t* parent;  // per binary internal node (CPT_WIDE_SAH only): its parent, arrivals, choice word
    uint32_t* arrive;
    uint32_t* choice;
    float* cost;       // C(n, 1..8)
};

size_t wide_scratch_layout(uint32_t leaves, bool sah, void* base, WideScratch* out)
{
    Carver c(base);
    WideScratch s;
    const size_t internal = std::max<uint32_t>(leaves - 1, 1u);
    s.queue = c.take<float4>(2 * internal);
    s.ctr = c.take<uint32_t>(kCtrWords);
    s.parent = sah ? c.take<uint32_t>(internal) : nullptr;
    s.arrive = sah ? c.take<uint32_t>(internal) : nullptr;
    s.choice = sah ? c.take<uint32_t>(internal) : nullptr;
    s.cost = sah ? c.take<float>(8 * internal) : nullptr;
    if (out) *out = s;
    return c.used();
}

__device__ __forceinline__ void read_record(const float4* __restrict__ bin, uint32_t b, float w[24])
{
    const float4* p = bin + 6 * (size_t)b;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const float4 f = p[k];
        w[4 * k] = f.x; w[4 * k + 1] = f.y; w[4 * k + 2] = f.z; w[4 * k + 3] = f.w;
    }
}

__device__ __forceinline__ float box_area(const float* b)
{
    const float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    return dx * dy + dy * dz + dz * dx;
}

// Child `side` of the binary node whose record is w and whose box is pb: its box and
// reference (internal: its binary index; leaf: parent * 2 + side | kLeafRef).
__device__ __forceinline__ void child_of(const float w[24], uint32_t parent, const float pb[6], int side, float box[6],
                                         uint32_t& ref)
{
    const uint32_t word = __float_as_uint(w[20]);
    const bool internal = side ? (word & 2u) : (word & 1u);
    const float* s = w + 10 * side;
    if (internal) {
#pragma unroll
        for (int k = 0; k < 6; ++k) box[k] = s[k];
        ref = side ? __float_as_uint(w[21]) : (word >> 2);
    } else {
        const float v0[3] = {s[0], s[1], s[2]};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float v1 = v0[a] + s[4 + a], v2 = v0[a] + s[7 + a];
            box[a] = fmaxf(fminf(fminf(v0[a], v1), v2), pb[a]);
            box[3 + a] = fminf(fmaxf(fmaxf(v0[a], v1), v2), pb[3 + a]);
            if (box[a] > box[3 + a]) box[a] = box[3 + a] = 0.5f * (box[a] + box[3 + a]);  // rounding: keep it a box
        }
        ref = (2u * parent + (uint32_t)side) | kLeafRef;
    }
}

// The root of the wide tree queued (level 0), the counters zeroed, the margin m.
__device__ void wide_init_tree(const float4* __restrict__ bin, float4* __restrict__ queue, uint32_t* __restrict__ ctr)
{
    float w[24];
    read_record(bin, 0, w);
    const uint32_t word = __float_as_uint(w[20]);
    float lo[3], hi[3], mag = 0.f;
    const float inf[6] = {-FLT_MAX, -FLT_MAX, -FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX};
    for (int a = 0; a < 3; ++a) { lo[a] = FLT_MAX; hi[a] = -FLT_MAX; }
    for (int side = 0; side < 2; ++side) {
        float b[6];
        uint32_t ref;
        child_of(w, 0, inf, side, b, ref);
        for (int a = 0; a < 3; ++a) { lo[a] = fminf(lo[a], b[a]); hi[a] = fmaxf(hi[a], b[3 + a]); }
    }
    (void)word;
    float diag2 = 0.f;
    for (int a = 0; a < 3; ++a) {
        mag = fmaxf(mag, fmaxf(fabsf(lo[a]), fabsf(hi[a])));
        diag2 += (hi[a] - lo[a]) * (hi[a] - lo[a]);
    }
    const float margin = ldexpf(mag + sqrtf(diag2), -20);
    queue[0] = make_float4(lo[0], lo[1], lo[2], __uint_as_float(0u));
    queue[1] = make_float4(hi[0], hi[1], hi[2], 0.f);
    ctr[0] = 1;  // wide nodes allocated: the root
    ctr[1] = 0;  // triangle records allocated
    ctr[2] = 0;  // blocks done in the current level
    ctr[3] = __float_as_uint(margin);
    for (int l = 0; l < kWideLevels + 2; ++l) ctr[4 + l] = l == 0 ? 0u : 1u;  // bounds[0] = 0, bounds[1] = 1
}

__global__ void k_wide_init(const float4* __restrict__ bin, float4* __restrict__ queue, uint32_t* __restrict__ ctr)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    wide_init_tree(bin, queue, ctr);
}

// Records a child of a wide node becomes: 1 for a binary leaf; for an internal binary
// node whose subtree has 2 or 3 leaves (up to kWideRecordLayers), that many — the child
// is then a leaf slot whose box holds those triangles; 0 for an internal child (a wide node).
__device__ __forceinline__ uint32_t leaf_records(const float4* __restrict__ bin, uint32_t ref, uint32_t bin_internal)
{
    if (ref & kLeafRef) return 1;
    if (kWideRecordLayers < 2 || ref >= bin_internal) return 0;
    const float4 f = bin[6 * (size_t)ref + 5];
    const uint32_t word = __float_as_uint(f.x);
    if (!(word & 3u)) return 2;  // both children leaves
    if ((word & 3u) == 3u || kWideRecordLayers < 3) return 0;
    const uint32_t d = (word & 1u) ? (word >> 2) : __float_as_uint(f.y);  // the internal child
    if (d >= bin_internal) return 0;
    return (__float_as_uint(bin[6 * (size_t)d + 5].x) & 3u) ? 0u : 3u;
}

// The triangle record of leaf `side` of binary node `parent`: the binary leaf slot's
// words (v0, index) (v1 - v0, 0) (v2 - v0, 0).
__device__ __forceinline__ void emit_leaf(const float4* __restrict__ bin, uint32_t parent, uint32_t side,
                                          float4* __restrict__ tr)
{
    const float2* sl = reinterpret_cast<const float2*>(bin + 6 * (size_t)parent) + 5 * side;
    const float2 a0 = sl[0], a1 = sl[1], a2 = sl[2], a3 = sl[3], a4 = sl[4];
    tr[0] = make_float4(a0.x, a0.y, a1.x, a1.y);  // v0, triangle index
    tr[1] = make_float4(a2.x, a2.y, a3.x, 0.f);   // v1 - v0
    tr[2] = make_float4(a3.y, a4.x, a4.y, 0.f);   // v2 - v0
}

// The cnt records (leaf_records) of child ref, in binary order: record j at rec + j * stride.
__device__ __forceinline__ void emit_records(const float4* __restrict__ bin, uint32_t ref, uint32_t cnt,
                                             float4* __restrict__ rec, size_t stride)
{
    const size_t st = 3 * stride;
    if (ref & kLeafRef) {
        emit_leaf(bin, (ref & ~kLeafRef) >> 1, ref & 1u, rec);
        return;
    }
    if (cnt == 2) {
        emit_leaf(bin, ref, 0, rec);
        emit_leaf(bin, ref, 1, rec + st);
        return;
    }
    const float4 f = bin[6 * (size_t)ref + 5];
    const uint32_t word = __float_as_uint(f.x);
    if (word & 1u) {  // side 0 is the two-leaf subtree
        const uint32_t d = word >> 2;
        emit_leaf(bin, d, 0, rec);
        emit_leaf(bin, d, 1, rec + st);
        emit_leaf(bin, ref, 1, rec + 2 * st);
    } else {
        const uint32_t d = __float_as_uint(f.y);
        emit_leaf(bin, ref, 0, rec);
        emit_leaf(bin, d, 0, rec + st);
        emit_leaf(bin, d, 1, rec + 2 * st);
    }
}

// Parents of the binary internal nodes and zeroed arrival counters (CPT_WIDE_SAH).
__global__ void k_sah_init(const float4* __restrict__ bin, uint32_t bin_internal, uint32_t* __restrict__ parent,
                           uint32_t* __restrict__ arrive)
{
    const uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= bin_internal) return;
    const float4 f = bin[6 * (size_t)n + 5];
    const uint32_t word = __float_as_uint(f.x), right = __float_as_uint(f.y);
    arrive[n] = 0;
    if (n == 0) parent[0] = CPT_INVALID_INDEX;  // the root (no node has it as a child)
    if (word == kUnusedNode) return;            // a record past the tree (split tree below its capacity)
    if ((word & 1u) && (word >> 2) < bin_internal) parent[word >> 2] = n;
    if ((word & 2u) && right < bin_internal) parent[right] = n;
}

// C(n, 1..8) and the choice word of binary internal node n from its children's (see
// CPT_WIDE_SAH); an internal child's table is final (its walk arrived before this one).
__device__ void sah_node(const float4* __restrict__ bin, uint32_t bin_internal, const uint32_t* __restrict__ parent,
                         uint32_t* __restrict__ choice, float* __restrict__ cost, uint32_t n)
{
    float w[24];
    read_record(bin, n, w);
    const uint32_t word = __float_as_uint(w[20]);
    // n's box: its slot in the parent's record, or for the root the union of its children
    float nb[6];
    const uint32_t p = parent[n];
    if (p < bin_internal) {
        const float* pr = reinterpret_cast<const float*>(bin + 6 * (size_t)p);
        const uint32_t pw = __float_as_uint(pr[20]);
        const int side = ((pw & 1u) && (pw >> 2) == n) ? 0 : 1;
        for (int k = 0; k < 6; ++k) nb[k] = pr[10 * side + k];
    } else {
        const float inf[6] = {-FLT_MAX, -FLT_MAX, -FLT_MAX, FLT_MAX, FLT_MAX, FLT_MAX};
        for (int a = 0; a < 3; ++a) { nb[a] = FLT_MAX; nb[3 + a] = -FLT_MAX; }
        for (int side = 0; side < 2; ++side) {
            float bx[6];
            uint32_t ref;
            child_of(w, n, inf, side, bx, ref);
            for (int a = 0; a < 3; ++a) { nb[a] = fminf(nb[a], bx[a]); nb[3 + a] = fmaxf(nb[3 + a], bx[3 + a]); }
        }
    }
    float tc[2][8];
    uint32_t pc[2];
    for (int side = 0; side < 2; ++side) {
        const bool internal = side ? (word & 2u) : (word & 1u);
        const uint32_t c = side ? __float_as_uint(w[21]) : (word >> 2);
        if (internal && c < bin_internal) {
            for (int i = 0; i < 8; ++i) tc[side][i] = __ldcg(cost + 8 * (size_t)c + i);
            pc[side] = sah_leaves(__ldcg(choice + c));
        } else {
            float bx[6];
            uint32_t ref;
            child_of(w, n, nb, side, bx, ref);
            const float leaf = box_area(bx) * kSahPrim;
            for (int i = 0; i < 8; ++i) tc[side][i] = leaf;
            pc[side] = 1;
        }
    }
    float d[9];
    uint32_t ch = 0;
    for (int j = 2; j <= 8; ++j) {
        float best = FLT_MAX;
        int bk = 1;
        for (int k = 1; k < j; ++k) {
            const float v = tc[0][k - 1] + tc[1][j - k - 1];
            if (v < best) { best = v; bk = k; }
        }
        d[j] = best;
        ch |= (uint32_t)bk << (8 + 3 * (j - 2));
    }
    const float area = box_area(nb);
    const uint32_t leaves = min(7u, pc[0] + pc[1]);
    const float c_node = area * kSahNode + d[8];
    const float c_leaf = leaves <= kWideRecordLayers ? area * kSahPrim * (float)leaves : FLT_MAX;
    ch |= leaves << 29;
    float c = c_node;
    if (c_leaf <= c_node) { c = c_leaf; ch |= 1u; }
    cost[8 * (size_t)n] = c;
    for (int j = 2; j <= 8; ++j) {
        if (d[j] < c) c = d[j];
        else ch |= 1u << (j - 1);
        cost[8 * (size_t)n + j - 1] = c;
    }
    choice[n] = ch;
}

// The cost tables bottom-up: a walk starts at every node with two leaf children and goes
// up while it is the last of a node's internal children to arrive (as the refit).
__global__ void k_sah_up(const float4* __restrict__ bin, uint32_t bin_internal, const uint32_t* __restrict__ parent,
                         uint32_t* __restrict__ arrive, uint32_t* __restrict__ choice, float* __restrict__ cost,
                         uint32_t* __restrict__ status)
{
    uint32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= bin_internal) return;
    if (__ldcg(status) & CPT_STATUS_TIMEOUT) return;  // no tree to walk (a sort gave up)
    if (__float_as_uint(bin[6 * (size_t)n + 5].x) & 3u) return;  // (kUnusedNode has both type bits)
    for (uint32_t steps = 0; steps < bin_internal; ++steps) {
        sah_node(bin, bin_internal, parent, choice, cost, n);
        const uint32_t p = parent[n];
        if (p >= bin_internal) return;  // the root
        __threadfence();
        const uint32_t need = __popc(__float_as_uint(bin[6 * (size_t)p + 5].x) & 3u);
        if (atomicAdd(&arrive[p], 1u) + 1u < need) return;
        __threadfence();
        n = p;
    }
    atomicOr(status, CPT_STATUS_BAD_INDEX);  // a cycle: not a tree
}

// Smallest e with ext <= 253 * 2^e (e in [-126, 127]): the 255 quanta of a byte less
// one quantum of slack on each side.
__device__ __forceinline__ int scale_exp(double ext)
{
    if (!(ext > 0.0)) return -126;
    int k;
    const double f = frexp(ext / 253.0, &k);  // ext / 253 = f * 2^k, f in [0.5, 1)
    int e = f > 0.5 ? k : k - 1;
    while (ldexp(253.0, e) < ext) ++e;
    return max(-126, min(127, e));
}

// The wide nodes [start, end) of one level: each collapses its binary subtree into up
// to 8 children, allocates its internal children (queued as the next level) and its
// leaf records.
__device__ __forceinline__ void wide_level_nodes(const float4* __restrict__ bin, float4* __restrict__ wide,
                                                 float4* __restrict__ tris, float4* __restrict__ queue,
                                                 uint32_t* __restrict__ ctr, uint32_t start, uint32_t end, float m,
                                                 uint32_t node_cap, uint32_t tri_cap, uint32_t bin_internal,
                                                 uint32_t* __restrict__ status, float (*s_box)[kWideBlock],
                                                 uint32_t (*s_ref)[kWideBlock],
                                                 const uint32_t* __restrict__ choice,  // null: the greedy collapse
                                                 uint32_t rot = 0)  // node start + j goes to thread (j + rot) mod T
{
    const int t = threadIdx.x;
    if (end > node_cap) {  // (only when the binary tree was not one: allocations past the cap were refused)
        if (blockIdx.x == 0 && t == 0) atomicOr(status, CPT_STATUS_BAD_INDEX);
        end = node_cap;
    }
    const uint32_t nt = gridDim.x * kWideBlock, tid = blockIdx.x * kWideBlock + t;
    const uint32_t first = (tid + nt - rot % nt) % nt;
    for (uint32_t wi = start + first; wi < end; wi += nt) {
        const float4 q0 = queue[2 * (size_t)wi], q1 = queue[2 * (size_t)wi + 1];
        const uint32_t b = __float_as_uint(q0.w);
        const float nb[6] = {q0.x, q0.y, q0.z, q1.x, q1.y, q1.z};
        if (b >= bin_internal) { atomicOr(status, CPT_STATUS_BAD_INDEX); continue; }
        int count = 0;
        if (choice) {
            // frontier: the binary node's children with the budgets of D(b, 8), then every
            // child whose budget (after the C(n, j) = C(n, j - 1) steps) is 2 or more is
            // replaced by its own two children with the budgets of its D(n, j)
            int budget[8];
            {
                float w[24];
                read_record(bin, b, w);
                const int k = sah_split(__ldcg(choice + b), 8);
                for (int side = 0; side < 2; ++side) {
                    float bx[6];
                    uint32_t ref;
                    child_of(w, b, nb, side, bx, ref);
                    for (int q = 0; q < 6; ++q) s_box[6 * count + q][t] = bx[q];
                    s_ref[count][t] = ref;
                    budget[count] = side ? 8 - k : k;
                    ++count;
                }
            }
            for (int i = 0; i < count;) {
                const uint32_t c = s_ref[i][t];
                if ((c & kLeafRef) || c >= bin_internal) { ++i; continue; }
                const uint32_t cc = __ldcg(choice + c);
                int j = budget[i];
                while (j >= 2 && sah_reduce(cc, j)) --j;
                if (j < 2 || count >= 8) { ++i; continue; }  // one child: a wide node or a leaf slot
                const int k = sah_split(cc, j);
                float pb[6];
                for (int q = 0; q < 6; ++q) pb[q] = s_box[6 * i + q][t];
                float w[24];
                read_record(bin, c, w);
                for (int side = 0; side < 2; ++side) {
                    float bx[6];
                    uint32_t ref;
                    child_of(w, c, pb, side, bx, ref);
                    const int slot = side == 0 ? i : count++;
                    for (int q = 0; q < 6; ++q) s_box[6 * slot + q][t] = bx[q];
                    s_ref[slot][t] = ref;
                    budget[slot] = side ? j - k : k;
                }
            }
        } else {
            // frontier: the binary node's children, then open the largest internal one
            {
                float w[24];
                read_record(bin, b, w);
                for (int side = 0; side < 2; ++side) {
                    float bx[6];
                    uint32_t ref;
                    child_of(w, b, nb, side, bx, ref);
                    for (int k = 0; k < 6; ++k) s_box[6 * count + k][t] = bx[k];
                    s_ref[count][t] = ref;
                    ++count;
                }
            }
            while (count < 8) {
                int best = -1;
                float best_area = -1.f;
                for (int i = 0; i < count; ++i) {
                    if (s_ref[i][t] & kLeafRef) continue;
                    float bx[6];
                    for (int k = 0; k < 6; ++k) bx[k] = s_box[6 * i + k][t];
                    const float a = box_area(bx);
                    if (a > best_area) { best_area = a; best = i; }
                }
                if (best < 0) break;
                const uint32_t c = s_ref[best][t];
                if (c >= bin_internal) { atomicOr(status, CPT_STATUS_BAD_INDEX); break; }
                float pb[6];
                for (int k = 0; k < 6; ++k) pb[k] = s_box[6 * best + k][t];
                float w[24];
                read_record(bin, c, w);
                for (int side = 0; side < 2; ++side) {
                    float bx[6];
                    uint32_t ref;
                    child_of(w, c, pb, side, bx, ref);
                    const int slot = side == 0 ? best : count++;
                    for (int k = 0; k < 6; ++k) s_box[6 * slot + k][t] = bx[k];
                    s_ref[slot][t] = ref;
                }
            }
        }
        // quantization frame
        float p[3];
        int e[3];
        double sc[3];
        float ctr_b[3];
        for (int a = 0; a < 3; ++a) {
            const double lo = (double)nb[a] - (double)m, hi = (double)nb[3 + a] + (double)m;
            e[a] = scale_exp((hi - lo) * (1.0 + 1e-6));
            sc[a] = ldexp(1.0, e[a]);
            // p one quantum below the widened box, rounded down to a float
            const double pd = lo - sc[a];
            float pf = (float)pd;
            if ((double)pf > pd) pf = nextafterf(pf, -FLT_MAX);
            p[a] = pf;
            ctr_b[a] = 0.5f * (nb[a] + nb[3 + a]);
        }
        // slots by direction: greedy smallest projection on the octant diagonal
        int slot_of[8];
        uint32_t used = 0, placed = 0;
        for (int i = 0; i < count; ++i) slot_of[i] = -1;
        for (int r = 0; r < count; ++r) {
            float best_c = FLT_MAX;
            int bi = 0, bs = 0;
            for (int i = 0; i < count; ++i) {
                if (placed >> i & 1u) continue;
                float c[3];
                for (int a = 0; a < 3; ++a) c[a] = 0.5f * (s_box[6 * i + a][t] + s_box[6 * i + 3 + a][t]) - ctr_b[a];
                for (int s = 0; s < 8; ++s) {
                    if (used >> s & 1u) continue;
                    const float cost = ((s & 1) ? -c[0] : c[0]) + ((s & 2) ? -c[1] : c[1]) + ((s & 4) ? -c[2] : c[2]);
                    if (cost < best_c) { best_c = cost; bi = i; bs = s; }
                }
            }
            slot_of[bi] = bs;
            placed |= 1u << bi;
            used |= 1u << bs;
        }
        // leaf slots (m1) and those holding a second (m2) and third (m3) record; the
        // node's records are layers of n_leaf records, one per leaf slot in slot order
        uint32_t cnt_of[8];
        uint32_t imask = 0, m1 = 0, m2 = 0, m3 = 0;
        for (int i = 0; i < count; ++i) {
            const uint32_t ref = s_ref[i][t];
            cnt_of[i] = (!choice || (ref & kLeafRef) || (ref < bin_internal && sah_leaf(__ldcg(choice + ref))))
                            ? leaf_records(bin, ref, bin_internal)
                            : 0u;
            const uint32_t bit = 1u << slot_of[i];
            if (!cnt_of[i]) imask |= bit;
            if (cnt_of[i] >= 1) m1 |= bit;
            if (cnt_of[i] >= 2) m2 |= bit;
            if (cnt_of[i] >= 3) m3 |= bit;
        }
        const uint32_t n_int = __popc(imask), n_leaf = __popc(m1);
        const uint32_t n_rec = n_leaf * (m3 ? 3u : m2 ? 2u : 1u);
        const uint32_t child_base = n_int ? atomicAdd(&ctr[0], n_int) : 0u;
        const uint32_t tri_base = n_rec ? atomicAdd(&ctr[1], n_rec) : 0u;
        if (child_base + n_int > node_cap || tri_base + n_rec > tri_cap) {
            atomicOr(status, CPT_STATUS_BAD_INDEX);
            continue;
        }
        // per axis, word j: slots 2j, 2j+1 as bytes (lo, hi, lo, hi); an empty slot is (255, 0)
        uint32_t qp[3][4];
        for (int a = 0; a < 3; ++a)
            for (int j = 0; j < 4; ++j) qp[a][j] = 0x00FF00FFu;
        for (int i = 0; i < count; ++i) {
            const int s = slot_of[i];
            const uint32_t ref = s_ref[i][t];
            float bx[6];
            for (int k = 0; k < 6; ++k) bx[k] = s_box[6 * i + k][t];
            for (int a = 0; a < 3; ++a) {
                // one quantum of slack each side for the traversal's folded plane offset
                const double lo = (double)bx[a] - (double)m, hi = (double)bx[3 + a] + (double)m;
                const int ql = (int)fmin(fmax(floor((lo - (double)p[a]) / sc[a]) - 1.0, 0.0), 255.0);
                const int qh = (int)fmin(fmax(ceil((hi - (double)p[a]) / sc[a]) + 1.0, 0.0), 255.0);
                const int sh = 16 * (s & 1);
                qp[a][s >> 1] = (qp[a][s >> 1] & ~(0xFFFFu << sh)) | (((uint32_t)ql | ((uint32_t)qh << 8)) << sh);
            }
            const uint32_t below = (1u << s) - 1u;
            if (cnt_of[i]) {
                emit_records(bin, ref, cnt_of[i], tris + 3 * (size_t)(tri_base + __popc(m1 & below)), n_leaf);
            } else {
                float4* qd = queue + 2 * (size_t)(child_base + __popc(imask & below));
                qd[0] = make_float4(bx[0], bx[1], bx[2], __uint_as_float(ref));
                qd[1] = make_float4(bx[3], bx[4], bx[5], 0.f);
            }
        }
        // the scale 2^e of an axis as the high half-word of its float bits: (e + 127) << 7
        const uint32_t hx = (uint32_t)(e[0] + 127) << 7, hy = (uint32_t)(e[1] + 127) << 7,
                       hz = (uint32_t)(e[2] + 127) << 7;
        float4* o = wide + 5 * (size_t)wi;
        o[0] = make_float4(p[0], p[1], p[2], __uint_as_float(hz | (imask << 24)));
        o[1] = make_float4(__uint_as_float(child_base), __uint_as_float(tri_base),
                           __uint_as_float(m1 | (m2 << 8) | (m3 << 16)), __uint_as_float(hx | (hy << 16)));
        for (int a = 0; a < 3; ++a)
            o[2 + a] = make_float4(__uint_as_float(qp[a][0]), __uint_as_float(qp[a][1]), __uint_as_float(qp[a][2]),
                                   __uint_as_float(qp[a][3]));
    }
}

// Every level in one cooperative launch: the blocks process a level's nodes and meet
// at a grid barrier (cooperative launch: all blocks are resident); the next level is
// what this one allocated, read by every thread between that barrier and a second one
// (so that no block allocates for the next level before every thread has read the
// same bound, and every block takes the same number of barriers). The walk stops at
// the first empty level, so a small tree costs its height in barriers, not kWideLevels
// launches. The last level bounds are left in ctr for k_wide_check (nodes still
// queued after kWideLevels levels: the tree was too tall).
__global__ void __launch_bounds__(kWideBlock) k_wide_levels(const float4* __restrict__ bin, float4* __restrict__ wide,
                                                            float4* __restrict__ tris, float4* __restrict__ queue,
                                                            uint32_t* __restrict__ ctr, uint32_t node_cap,
                                                            uint32_t tri_cap, uint32_t bin_internal,
                                                            uint32_t* __restrict__ status,
                                                            const uint32_t* __restrict__ choice)
{
    __shared__ float s_box[8 * 6][kWideBlock];
    __shared__ uint32_t s_ref[8][kWideBlock];
    // A sort of the build (or of the split tree) gave up a look-back wait: the binary
    // tree is not one. Every block leaves at once (the word was set before this launch,
    // so all see it and none waits at the barrier), and no node is written.
    if (__ldcg(status) & CPT_STATUS_TIMEOUT) return;
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const float m = __uint_as_float(__ldcg(&ctr[3]));
    uint32_t start = 0, end = 1;  // level 0: the root, queued by k_wide_init
    int level = 0;
    for (; level < kWideLevels && start < end; ++level) {
        wide_level_nodes(bin, wide, tris, queue, ctr, start, end, m, node_cap, tri_cap, bin_internal, status, s_box,
                         s_ref, choice);
        grid.sync();
        const uint32_t next = __ldcg(&ctr[0]);  // every node allocated so far: final after the barrier
        grid.sync();
        start = end;
        end = next;
    }
    if (grid.thread_rank() == 0) {
        ctr[4 + kWideLevels] = start;
        ctr[4 + kWideLevels + 1] = end;
    }
}

__global__ void k_wide_check(const uint32_t* __restrict__ ctr, uint32_t* __restrict__ status,
                             uint32_t* __restrict__ counts_out)
{
    if (threadIdx.x != 0) return;
    // nodes allocated by the last level were never filled: the tree was too tall
    if (ctr[4 + kWideLevels + 1] != ctr[4 + kWideLevels]) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
    if (counts_out) { counts_out[0] = ctr[0]; counts_out[1] = ctr[1]; }
}

// ---- batched wide build: the wide trees of several binary trees in one cooperative
// launch, every level of every tree between the same grid barriers ----
constexpr uint32_t kWideBatchMax = CPT_MAX_BATCH_SCENES;
struct WideBatchTree {
    const float4* bin;
    float4* wide;
    float4* tris;
    float4* queue;
    uint32_t* ctr;
    uint32_t* status;
    uint32_t node_cap, tri_cap, bin_internal;
};
struct WideBatch {  // passed by value: a call can be captured in a CUDA graph
    WideBatchTree t[kWideBatchMax];
    uint32_t count;
    uint32_t* bounds;  // per tree: the current level's [start, end)
};

__global__ void k_wide_init_batch(WideBatch wb)
{
    if (threadIdx.x != 0 || blockIdx.x >= wb.count) return;
    const WideBatchTree& T = wb.t[blockIdx.x];
    wide_init_tree(T.bin, T.queue, T.ctr);
    wb.bounds[2 * blockIdx.x] = 0;  // level 0: the root
    wb.bounds[2 * blockIdx.x + 1] = 1;
}

// As k_wide_levels, over every tree of the batch: a level's nodes of all trees are
// numbered one after the other (tree by tree), and node g of that numbering goes to
// thread g mod (threads of the grid), so the work is shared out whatever the trees'
// sizes. Block 0 moves every tree to its next level between the two barriers.
__global__ void __launch_bounds__(kWideBlock) k_wide_levels_batch(WideBatch wb)
{
    __shared__ float s_box[8 * 6][kWideBlock];
    __shared__ uint32_t s_ref[8][kWideBlock];
    __shared__ uint32_t s_start[kWideBatchMax], s_end[kWideBatchMax], s_rot[kWideBatchMax + 1];
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const uint32_t n = min(wb.count, kWideBatchMax);
    int level = 0;
    for (; level < kWideLevels; ++level) {
        if (threadIdx.x < n) {
            const WideBatchTree& T = wb.t[threadIdx.x];
            const bool skip = __ldcg(T.status) & CPT_STATUS_TIMEOUT;  // (set before the launch: every block agrees)
            s_start[threadIdx.x] = __ldcg(wb.bounds + 2 * threadIdx.x);
            s_end[threadIdx.x] = skip ? s_start[threadIdx.x] : __ldcg(wb.bounds + 2 * threadIdx.x + 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (uint32_t i = 0; i < n; ++i) {
                s_rot[i] = acc;
                acc += s_end[i] > s_start[i] ? s_end[i] - s_start[i] : 0u;
            }
            s_rot[n] = acc;
        }
        __syncthreads();
        if (s_rot[n] == 0) break;  // every tree done (the same bounds in every block)
        for (uint32_t i = 0; i < n; ++i) {
            if (s_end[i] <= s_start[i]) continue;
            const WideBatchTree& T = wb.t[i];
            wide_level_nodes(T.bin, T.wide, T.tris, T.queue, T.ctr, s_start[i], s_end[i],
                             __uint_as_float(__ldcg(&T.ctr[3])), T.node_cap, T.tri_cap, T.bin_internal, T.status,
                             s_box, s_ref, nullptr, s_rot[i]);
        }
        grid.sync();
        if (blockIdx.x == 0 && threadIdx.x < n) {  // every node allocated so far: final after the barrier
            wb.bounds[2 * threadIdx.x] = s_end[threadIdx.x];
            wb.bounds[2 * threadIdx.x + 1] = __ldcg(&wb.t[threadIdx.x].ctr[0]);
        }
        grid.sync();
    }
    if (blockIdx.x == 0 && threadIdx.x < n && !(__ldcg(wb.t[threadIdx.x].status) & CPT_STATUS_TIMEOUT)) {
        const WideBatchTree& T = wb.t[threadIdx.x];  // the last bounds, for k_wide_check_batch
        T.ctr[4 + kWideLevels] = __ldcg(wb.bounds + 2 * threadIdx.x);
        T.ctr[4 + kWideLevels + 1] = __ldcg(wb.bounds + 2 * threadIdx.x + 1);
    }
}

__global__ void k_wide_check_batch(WideBatch wb)
{
    const uint32_t i = threadIdx.x;
    if (i >= wb.count) return;
    const WideBatchTree& T = wb.t[i];
    if (T.ctr[4 + kWideLevels + 1] != T.ctr[4 + kWideLevels]) atomicOr(T.status, CPT_STATUS_STACK_OVERFLOW);
    T.status[2] = T.ctr[0];
    T.status[3] = T.ctr[1];
}

}  // namespace
}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_lbvh_wide_bytes(uint32_t leaves, uint32_t flags, size_t* node_bytes, size_t* tri_bytes)
{
    if (flags & ~CPT_WIDE_SAH) return 0;
    if (leaves < 2 || leaves > 0xFFFFFFFFu / kWideRecordLayers) return 0;
    if (node_bytes) *node_bytes = align_up((size_t)(leaves - 1) * 80, 256);
    if (tri_bytes) *tri_bytes = align_up((size_t)leaves * kWideRecordLayers * 48, 256);
    return wide_scratch_layout(leaves, flags & CPT_WIDE_SAH, nullptr, nullptr);
}

extern "C" int cpt_lbvh_wide(cpt_bvh* bvh, uint32_t flags, void* nodes, size_t node_bytes, void* tris,
                             size_t tri_bytes, void* scratch, size_t scratch_bytes, cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_wide");
    if (!bvh || !bvh->nodes || !bvh->status || !nodes || !tris || !scratch) return CPT_ERR_INVALID_ARGUMENT;
    const bool split = bvh->split_nodes != nullptr;
    const uint32_t leaves = split ? bvh->split_capacity : bvh->n;
    size_t nb = 0, tb = 0;
    const size_t need = cpt_lbvh_wide_bytes(leaves, flags, &nb, &tb);
    if (!need) return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < need || node_bytes < nb || tri_bytes < tb) return CPT_ERR_SCRATCH_TOO_SMALL;
    if ((reinterpret_cast<uintptr_t>(nodes) & 15) || (reinterpret_cast<uintptr_t>(tris) & 15) ||
        (reinterpret_cast<uintptr_t>(scratch) & 255))
        return CPT_ERR_INVALID_ARGUMENT;
    bvh->wide_nodes = nullptr;
    bvh->wide_tris = nullptr;
    bvh->wide_capacity = 0;
    WideScratch ws;
    const bool sah = flags & CPT_WIDE_SAH;
    wide_scratch_layout(leaves, sah, scratch, &ws);
    const float4* bin = static_cast<const float4*>(split ? bvh->split_nodes : bvh->nodes);
    k_wide_init<<<1, 32, 0, stream>>>(bin, ws.queue, ws.ctr);
    CPT_LAUNCH_CHECK();
    if (sah) {
        const uint32_t internal = leaves - 1;
        const unsigned g = (internal + 255) / 256;
        k_sah_init<<<g, 256, 0, stream>>>(bin, internal, ws.parent, ws.arrive);
        CPT_LAUNCH_CHECK();
        k_sah_up<<<g, 256, 0, stream>>>(bin, internal, ws.parent, ws.arrive, ws.choice, ws.cost, bvh->status);
        CPT_LAUNCH_CHECK();
    }
    // one cooperative launch over every level: as many blocks as the largest level can
    // use, no more than can be resident at once
    static int occ[64] = {0};
    int dev = 0;
    CPT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CPT_ERR_INVALID_ARGUMENT;
    if (!occ[dev]) {
        int o = 0;
        CPT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_wide_levels, kWideBlock, 0));
        occ[dev] = std::max(1, o);
    }
    const uint64_t widest = std::min<uint64_t>((uint64_t)leaves - 1, (uint64_t)sm_count() * occ[dev] * kWideBlock);
    const int blocks = (int)std::max<uint64_t>(1, (widest + kWideBlock - 1) / kWideBlock);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kWideBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // (also as a node of a captured graph)
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CPT_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_wide_levels, bin, static_cast<float4*>(nodes), static_cast<float4*>(tris),
                                    ws.queue, ws.ctr, leaves - 1, leaves * kWideRecordLayers, leaves - 1, bvh->status,
                                    static_cast<const uint32_t*>(ws.choice)));
    note_launch();
    k_wide_check<<<1, 32, 0, stream>>>(ws.ctr, bvh->status, bvh->status + 2);
    CPT_LAUNCH_CHECK();
    bvh->wide_nodes = nodes;
    bvh->wide_tris = tris;
    bvh->wide_capacity = leaves;
    return CPT_OK;
}

extern "C" size_t cpt_lbvh_wide_batch_scratch_bytes(const uint32_t* leaves, uint32_t trees)
{
    if (!leaves || trees < 1 || trees > kWideBatchMax) return 0;
    size_t total = align_up(2 * sizeof(uint32_t) * kWideBatchMax, 256);  // the level bounds
    for (uint32_t i = 0; i < trees; ++i) {
        const size_t one = cpt_lbvh_wide_bytes(leaves[i], 0, nullptr, nullptr);
        if (!one) return 0;
        total += one;
    }
    return total;
}

extern "C" int cpt_lbvh_wide_batch(cpt_bvh* const* bvhs, uint32_t trees, void* const* nodes, const size_t* node_bytes,
                                   void* const* tris, const size_t* tri_bytes, void* scratch, size_t scratch_bytes,
                                   cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_wide_batch");
    if (!bvhs || !nodes || !node_bytes || !tris || !tri_bytes || !scratch || trees < 1 || trees > kWideBatchMax)
        return CPT_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(scratch) & 255) return CPT_ERR_INVALID_ARGUMENT;
    WideBatch wb = {};
    wb.count = trees;
    char* base = static_cast<char*>(scratch);
    size_t off = align_up(2 * sizeof(uint32_t) * kWideBatchMax, 256);
    wb.bounds = reinterpret_cast<uint32_t*>(base);
    uint64_t total_internal = 0;
    for (uint32_t i = 0; i < trees; ++i) {
        cpt_bvh* bvh = bvhs[i];
        if (!bvh || !bvh->nodes || !bvh->status || !nodes[i] || !tris[i]) return CPT_ERR_INVALID_ARGUMENT;
        if ((reinterpret_cast<uintptr_t>(nodes[i]) & 15) || (reinterpret_cast<uintptr_t>(tris[i]) & 15))
            return CPT_ERR_INVALID_ARGUMENT;
        const bool split = bvh->split_nodes != nullptr;
        const uint32_t leaves = split ? bvh->split_capacity : bvh->n;
        size_t nb = 0, tb = 0;
        const size_t one = cpt_lbvh_wide_bytes(leaves, 0, &nb, &tb);
        if (!one) return CPT_ERR_INVALID_ARGUMENT;
        if (node_bytes[i] < nb || tri_bytes[i] < tb || off + one > scratch_bytes) return CPT_ERR_SCRATCH_TOO_SMALL;
        WideScratch ws;
        wide_scratch_layout(leaves, false, base + off, &ws);
        off += one;
        WideBatchTree& T = wb.t[i];
        T.bin = static_cast<const float4*>(split ? bvh->split_nodes : bvh->nodes);
        T.wide = static_cast<float4*>(nodes[i]);
        T.tris = static_cast<float4*>(tris[i]);
        T.queue = ws.queue;
        T.ctr = ws.ctr;
        T.status = bvh->status;
        T.node_cap = leaves - 1;
        T.tri_cap = leaves * kWideRecordLayers;
        T.bin_internal = leaves - 1;
        total_internal += leaves - 1;
    }
    for (uint32_t i = 0; i < trees; ++i) {
        bvhs[i]->wide_nodes = nullptr;
        bvhs[i]->wide_tris = nullptr;
        bvhs[i]->wide_capacity = 0;
    }
    k_wide_init_batch<<<trees, 32, 0, stream>>>(wb);
    CPT_LAUNCH_CHECK();
    static int occ[64] = {0};
    int dev = 0;
    CPT_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CPT_ERR_INVALID_ARGUMENT;
    if (!occ[dev]) {
        int o = 0;
        CPT_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, k_wide_levels_batch, kWideBlock, 0));
        occ[dev] = std::max(1, o);
    }
    const uint64_t widest = std::min<uint64_t>(total_internal, (uint64_t)sm_count() * occ[dev] * kWideBlock);
    const int blocks = (int)std::max<uint64_t>(1, (widest + kWideBlock - 1) / kWideBlock);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kWideBlock);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CPT_CUDA_TRY(cudaLaunchKernelEx(&cfg, k_wide_levels_batch, wb));
    note_launch();
    k_wide_check_batch<<<1, kWideBatchMax, 0, stream>>>(wb);
    CPT_LAUNCH_CHECK();
    for (uint32_t i = 0; i < trees; ++i) {
        cpt_bvh* bvh = bvhs[i];
        bvh->wide_nodes = nodes[i];
        bvh->wide_tris = tris[i];
        bvh->wide_capacity = bvh->split_nodes ? bvh->split_capacity : bvh->n;
    }
    return CPT_OK;
}
