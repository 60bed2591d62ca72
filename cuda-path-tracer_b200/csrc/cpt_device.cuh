// Device-side arithmetic shared by the build, traversal and render kernels.
//
// Every floating-point operation that feeds a result compared with the
// reference is written with a round-to-nearest intrinsic (__fadd_rn, __fmul_rn,
// ...), which nvcc never contracts into an FMA. That reproduces the operation
// sequence of the reference's glm expressions exactly:
//   glm::min(x, y) = x < y ? x : y,  glm::max(x, y) = x > y ? x : y   (func_common.inl:15-26)
//   dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z                          (func_geometric.inl:54-61)
//   cross, normalize(v) = v * (1 / sqrt(dot(v, v)))                    (func_geometric.inl:74-96)
//   mix(x, y, a) = x + a * (y - x)                                     (func_common.inl:143-151)
// so Morton codes, boxes, hit distances and shaded radiance are bit-identical to
// a no-contraction build of the reference.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <float.h>

namespace cpt {

struct f3 { float x, y, z; };

__device__ __forceinline__ f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ f3 add(f3 a, f3 b) { return mk3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)); }
__device__ __forceinline__ f3 sub(f3 a, f3 b) { return mk3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ f3 mul(f3 a, f3 b) { return mk3(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)); }
__device__ __forceinline__ f3 muls(f3 a, float s) { return mk3(__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)); }
__device__ __forceinline__ f3 neg(f3 a) { return mk3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(f3 a, f3 b)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ f3 cross(f3 a, f3 b)
{
    return mk3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(b.y, a.z)),
               __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(b.z, a.x)),
               __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(b.x, a.y)));
}
__device__ __forceinline__ f3 normalize(f3 v) { return muls(v, __frcp_rn(__fsqrt_rn(dot(v, v)))); }
__device__ __forceinline__ f3 mix3(f3 x, f3 y, float a) { return add(x, muls(sub(y, x), a)); }
// barycentricLerp (math_util.h:19-23): v0*(1-u-v) + v1*u + v2*v
__device__ __forceinline__ f3 bary(f3 a, f3 b, f3 c, float u, float v)
{
    float w = __fsub_rn(__fsub_rn(1.0f, u), v);
    return add(add(muls(a, w), muls(b, u)), muls(c, v));
}
__device__ __forceinline__ float gmin(float x, float y) { return x < y ? x : y; }
__device__ __forceinline__ float gmax(float x, float y) { return x > y ? x : y; }
__device__ __forceinline__ f3 ld3(const float* p) { return mk3(p[0], p[1], p[2]); }
__device__ __forceinline__ f3 xyz(float4 v) { return mk3(v.x, v.y, v.z); }

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11). Replaces the reference's per-thread curand XORWOW
// (cuda_path_tracer.cu:400-402) with a counter-based stream:
//   bounce i of pixel p, global sample f : counter (p, f, i, 0)
//   camera jitter of global sample f     : counter (~0, f, 0, 1)
//   uniform from a word w                : (w >> 8) * 2^-24 in [0, 1)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        uint4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}
__device__ __forceinline__ float u01(uint32_t w) { return __fmul_rn(__uint2float_rn(w >> 8), 1.0f / 16777216.0f); }

// sin(2*pi*u), cos(2*pi*u). The reference takes sinf/cosf of CUDA_2PI * u
// (random.h:97-113); here the argument is reduced exactly in turns (quarter-turn
// index and fraction, exact in binary floating point), folded to an eighth of a
// turn, and sine/cosine of (pi/2)*g, g in [0, 1/2], are the Taylor series to
// degree 9 / 10 (truncation below 2e-9) in Horner form with fused multiply-adds —
// correctly rounded operations, so host and device agree to the bit.
__device__ __forceinline__ void sincos_turns(float u, float* s_out, float* c_out)
{
    const float S1 = 1.5707963705062866f, S3 = -0.6459640860557556f, S5 = 0.07969262450933456f,
                S7 = -0.004681753925979137f, S9 = 0.00016044118092395365f;
    const float C2 = -1.2337005138397217f, C4 = 0.25366950035095215f, C6 = -0.020863480865955353f,
                C8 = 0.0009192602592520416f, C10 = -2.520204179745633e-05f;
    float t = __fmul_rn(u, 4.0f);
    float q = floorf(t);
    float f = __fsub_rn(t, q);
    int quad = ((int)q) & 3;
    bool fold = f > 0.5f;
    float g = fold ? __fsub_rn(1.0f, f) : f;
    float g2 = __fmul_rn(g, g);
    float sp = __fmaf_rn(g2, S9, S7);
    sp = __fmaf_rn(g2, sp, S5);
    sp = __fmaf_rn(g2, sp, S3);
    sp = __fmaf_rn(g2, sp, S1);
    float sg = __fmul_rn(g, sp);
    float cp = __fmaf_rn(g2, C10, C8);
    cp = __fmaf_rn(g2, cp, C6);
    cp = __fmaf_rn(g2, cp, C4);
    cp = __fmaf_rn(g2, cp, C2);
    float cg = __fmaf_rn(g2, cp, 1.0f);
    float sa = fold ? cg : sg, ca = fold ? sg : cg;
    float s, c;
    switch (quad) {
        case 0: s = sa; c = ca; break;
        case 1: s = ca; c = -sa; break;
        case 2: s = -sa; c = -ca; break;
        default: s = -ca; c = sa; break;
    }
    *s_out = s;
    *c_out = c;
}

// Warp-aggregated append: one atomic per warp, lanes get consecutive slots in
// lane order. Returns this lane's slot (only meaningful when pred is true).
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool pred)
{
    unsigned active = __activemask();
    unsigned mask = __ballot_sync(active, pred);
    if (!pred) return 0;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void warp_count_u64(unsigned long long* counter, uint32_t v)
{
    if (!counter) return;
    unsigned active = __activemask();
    uint32_t sum = __reduce_add_sync(active, v);
    if ((threadIdx.x & 31) == (uint32_t)(__ffs(active) - 1) && sum) atomicAdd(counter, (unsigned long long)sum);
}

}  // namespace cpt
