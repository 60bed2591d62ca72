// Radiance cache (cpt_rc_*): an MLP trained online on the path suffixes the tracer
// itself generates, queried at each path's secondary vertex instead of tracing
// the rest of the path.
//
// Estimator. The reference's sample of a depth-(B+1) path (blinnPhongShadingPathTrace,
// cuda_path_tracer.cu:245-333) is
//     E0 + I a0 a1 (L1 + T),   T = a2 L2 + a2 a3 L3 + ... + (a2..aB) LB,
// with ak the albedo and Lk the light gathered at vertex k, I the indirect
// intensity. The cached render traces vertices 0 and 1 exactly as the plain tracer
// (same random stream, so the same first bounce) and replaces T by the network's
// prediction C(x1, d1, n1, a1) >= 0; T depends on vertex 1 alone, so the emission
// and direct light at vertex 1 stay exact and only the multi-bounce remainder is
// approximated.
//
// Training. Every frame a second, independent set of full-depth paths (about
// cpt_rc_params.train_samples of them, one per pixel of a reduced-resolution copy
// of each view) records (x1, d1, n1, a1), the weight W1 = I a0 a1 and the radiance
// R1 after vertex 1; when the path ends, T = (R - R1) / W1 is its training target.
// The samples are split into train_steps batches; each batch is one fused
// forward/backward pass (k_rc_train: per-block partial weight gradients) followed
// by Adam (k_rc_adam: sums the partials, updates FP32 master weights, writes the
// BF16 copies for training and for inference, the latter optionally an exponential
// moving average). Loss: relative L2, (y - t)^2 / (y^2 + 0.01) with y held constant
// in the denominator (Mueller et al., "Real-time Neural Radiance Caching for Path
// Tracing", SIGGRAPH 2021).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>
#include <algorithm>
#include <mutex>
#include <new>
#include <vector>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"
#include "rc_mlp.cuh"
#include "render_hook.h"

namespace cpt {
namespace rc {

using bf16 = __nv_bfloat16;

constexpr int kTrainWarps = 8;
constexpr int kTrainRows = 16 * kTrainWarps;
constexpr int kTrainBlock = 32 * kTrainWarps;
constexpr int kMaxTrainBlocks = 512;
constexpr int kInferWarps = 8;
constexpr int kInferBlock = 32 * kInferWarps;
constexpr float kLossEps = 0.01f;

constexpr size_t kTrainSmem = sizeof(bf16) * ((size_t)kWSmem + (size_t)kTrainRows * kXS + 6ull * kTrainRows * kAS +
                                              (size_t)kTrainRows * kZS);
constexpr size_t kInferSmem = sizeof(bf16) * ((size_t)kWSmem + (size_t)kInferWarps * 16 * kXS);

__device__ __forceinline__ void box_params(const float* box, float (&bmin)[3], float (&binv)[3])
{
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        bmin[a] = box[a];
        const float ext = box[3 + a] - box[a];
        binv[a] = ext > 0.f ? 1.0f / ext : 0.f;
    }
}

__device__ __forceinline__ void batch_range(const uint32_t* count_dev, uint32_t count_host, uint32_t step,
                                            uint32_t steps, uint32_t& lo, uint32_t& hi)
{
    const uint32_t n = count_dev ? *count_dev : count_host;
    lo = (uint32_t)((uint64_t)n * step / steps);
    hi = (uint32_t)((uint64_t)n * (step + 1) / steps);
}

// ---------------------------------------------------------------------------
// inference

// kRecords = false: `in` holds samples (4 float4 each), out[i] = (rgb, 0).
// kRecords = true: `in` holds render records (5 float4 each: position | path id,
// direction | W.x, normal | W.y, albedo | W.z, R1); the path's radiance in `out`
// (the wavefront state, 2 float4 per path) gains W * max(prediction, 0).
template <bool kRecords>
__global__ void __launch_bounds__(kInferBlock) k_rc_infer(const bf16* __restrict__ w, const float4* __restrict__ in,
                                                          const uint32_t* __restrict__ count_dev, uint32_t count_host,
                                                          const float* __restrict__ box, float4* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* ws = reinterpret_cast<bf16*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    bf16* xw = ws + kWSmem + warp * 16 * kXS;
    load_weights(w, ws);
    float bmin[3], binv[3];
    box_params(box, bmin, binv);
    __syncthreads();
    const uint32_t n = count_dev ? *count_dev : count_host;
    const uint32_t tiles = (n + 15) / 16;
    constexpr int kF4 = kRecords ? kRecordF4 : kSampleF4;
    for (uint32_t t = blockIdx.x * kInferWarps + warp; t < tiles; t += gridDim.x * kInferWarps) {
        const uint32_t base = t * 16;
        const int r = lane & 15;
        const uint32_t gi = base + r;
        const bool valid = gi < n;
        float4 f[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = valid ? in[(size_t)kF4 * gi + k] : make_float4(0.f, 0.f, 0.f, 0.f);
        encode_half(f, valid, bmin, binv, lane >> 4, xw + r * kXS);
        __syncwarp();
        float y[2][4];
        forward16(ws, xw, 0, nullptr, y, lane);
        // row (lane >> 2) and row + 8: columns 2q, 2q+1 of n-tile 0; blue is lane+1's first column
        const float b0 = __shfl_down_sync(0xFFFFFFFFu, y[0][0], 1);
        const float b1 = __shfl_down_sync(0xFFFFFFFFu, y[0][2], 1);
        if ((lane & 3) == 0) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t row = base + (lane >> 2) + 8 * h;
                if (row >= n) continue;
                const float pr = y[0][2 * h], pg = y[0][2 * h + 1], pb = h ? b1 : b0;
                if (kRecords) {
                    const float4 r0 = in[(size_t)kF4 * row], r1 = in[(size_t)kF4 * row + 1];
                    const float4 r2 = in[(size_t)kF4 * row + 2], r3 = in[(size_t)kF4 * row + 3];
                    const uint32_t pid = __float_as_uint(r0.w);
                    float4 acc = out[2 * (size_t)pid];
                    acc.x = __fadd_rn(acc.x, __fmul_rn(r1.w, fmaxf(pr, 0.f)));
                    acc.y = __fadd_rn(acc.y, __fmul_rn(r2.w, fmaxf(pg, 0.f)));
                    acc.z = __fadd_rn(acc.z, __fmul_rn(r3.w, fmaxf(pb, 0.f)));
                    out[2 * (size_t)pid] = acc;
                } else {
                    out[row] = make_float4(pr, pg, pb, 0.f);
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// training

// dZ_{l-1} for the warp's 16 rows: (dZ_l W_l^T) masked by ReLU'(activation l-1).
template <int kK>
__device__ __forceinline__ void back16(const bf16* dzl, int dz_stride, const bf16* wl, int wst, const bf16* act_prev,
                                       bf16* dz_out, int r0, int lane)
{
    float acc[8][4];
#pragma unroll
    for (int n = 0; n < 8; ++n) acc[n][0] = acc[n][1] = acc[n][2] = acc[n][3] = 0.f;
#pragma unroll
    for (int kt = 0; kt < kK / 16; ++kt) {
        uint32_t a[4];
        ldsm_x4(a, frag_a(dzl, dz_stride, r0, 16 * kt, lane));
#pragma unroll
        for (int np = 0; np < 4; ++np) {
            uint32_t b[4];
            ldsm_x4(b, frag_bt(wl, wst, 16 * kt, 16 * np, lane));
            mma_bf16(acc[2 * np], a, b[0], b[1]);
            mma_bf16(acc[2 * np + 1], a, b[2], b[3]);
        }
    }
    const int r = r0 + (lane >> 2), c = 2 * (lane & 3);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float2 m0 = unpack_bf16(*reinterpret_cast<const uint32_t*>(act_prev + r * kAS + 8 * nt + c));
        const float2 m1 = unpack_bf16(*reinterpret_cast<const uint32_t*>(act_prev + (r + 8) * kAS + 8 * nt + c));
        *reinterpret_cast<uint32_t*>(dz_out + r * kAS + 8 * nt + c) =
            pack_bf16(m0.x > 0.f ? acc[nt][0] : 0.f, m0.y > 0.f ? acc[nt][1] : 0.f);
        *reinterpret_cast<uint32_t*>(dz_out + (r + 8) * kAS + 8 * nt + c) =
            pack_bf16(m1.x > 0.f ? acc[nt][2] : 0.f, m1.y > 0.f ? acc[nt][3] : 0.f);
    }
}

// dW_l += S^T dZ_l over the chunk's kTrainRows rows for the warp's kUnits
// m16 x n8 tiles (unit u = warp + 8k; tile (u / ntiles, u % ntiles)).
template <int kUnits>
__device__ __forceinline__ void dw_layer(const bf16* s, int s_stride, const bf16* dzl, int dz_stride, int ntiles,
                                         float (*acc)[4], int warp, int lane)
{
#pragma unroll
    for (int k = 0; k < kUnits; ++k) {
        const int u = warp + kTrainWarps * k;
        const int mt = u / ntiles, nt = u - mt * ntiles;
#pragma unroll
        for (int ks = 0; ks < kTrainRows / 16; ++ks) {
            uint32_t a[4], b[2];
            ldsm_x4_t(a, frag_at(s, s_stride, 16 * mt, 16 * ks, lane));
            ldsm_x2_t(b, frag_b(dzl, dz_stride, 16 * ks, 8 * nt, lane));
            mma_bf16(acc[k], a, b[0], b[1]);
        }
    }
}

template <int kUnits>
__device__ __forceinline__ void write_units(float* p, int l, const float (*acc)[4], int warp, int lane)
{
    const int ntiles = fan_out(l) / 8, fo = fan_out(l);
    float* pl = p + param_off(l);
#pragma unroll
    for (int k = 0; k < kUnits; ++k) {
        const int u = warp + kTrainWarps * k;
        const int mt = u / ntiles, nt = u - mt * ntiles;
        const int m = 16 * mt + (lane >> 2), n = 8 * nt + 2 * (lane & 3);
        *reinterpret_cast<float2*>(pl + m * fo + n) = make_float2(acc[k][0], acc[k][1]);
        *reinterpret_cast<float2*>(pl + (m + 8) * fo + n) = make_float2(acc[k][2], acc[k][3]);
    }
}

// Units per warp and layer: layer 0 (96x64) 48 tiles, layers 1-3 (64x64) 32, layer 4 (64x16) 8.
constexpr int kU0 = (kIn / 16) * (kHid / 8) / kTrainWarps;
constexpr int kU1 = (kHid / 16) * (kHid / 8) / kTrainWarps;
constexpr int kU4 = (kHid / 16) * (kOut / 8) / kTrainWarps;
static_assert(kU0 == 6 && kU1 == 4 && kU4 == 1, "tile split");

__global__ void __launch_bounds__(kTrainBlock, 1) k_rc_train(const bf16* __restrict__ w,
                                                             const float4* __restrict__ samples,
                                                             const uint32_t* __restrict__ count_dev,
                                                             uint32_t count_host, uint32_t step, uint32_t steps,
                                                             const float* __restrict__ box,
                                                             float* __restrict__ partials, float* __restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    bf16* ws = reinterpret_cast<bf16*>(smem_raw);
    bf16* xs = ws + kWSmem;
    bf16* act0 = xs + kTrainRows * kXS;
    bf16* acts[4] = {act0, act0 + kTrainRows * kAS, act0 + 2 * kTrainRows * kAS, act0 + 3 * kTrainRows * kAS};
    bf16* dz[2] = {act0 + 4 * kTrainRows * kAS, act0 + 5 * kTrainRows * kAS};
    bf16* dz4 = act0 + 6 * kTrainRows * kAS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r0 = 16 * warp;
    load_weights(w, ws);
    float bmin[3], binv[3];
    box_params(box, bmin, binv);
    uint32_t lo, hi;
    batch_range(count_dev, count_host, step, steps, lo, hi);
    const uint32_t batch = hi - lo;
    const float inv_batch = batch ? 1.0f / (float)batch : 0.f;
    float g4[kU4][4], g3[kU1][4], g2[kU1][4], g1[kU1][4], g0[kU0][4];
#define CPT_ZERO(a, n) \
    for (int k_ = 0; k_ < n; ++k_) a[k_][0] = a[k_][1] = a[k_][2] = a[k_][3] = 0.f
    CPT_ZERO(g4, kU4); CPT_ZERO(g3, kU1); CPT_ZERO(g2, kU1); CPT_ZERO(g1, kU1); CPT_ZERO(g0, kU0);
#undef CPT_ZERO
    float loss_sum = 0.f;
    const uint32_t chunks = (batch + kTrainRows - 1) / kTrainRows;
    for (uint32_t ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
        __syncthreads();  // weights loaded; the previous chunk's readers are done
        const uint32_t base = lo + ch * kTrainRows;
        {
            const int r = r0 + (lane & 15);
            const uint32_t gi = base + r;
            const bool valid = gi < hi;
            float4 f[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) f[k] = valid ? samples[4 * (size_t)gi + k] : make_float4(0.f, 0.f, 0.f, 0.f);
            encode_half(f, valid, bmin, binv, lane >> 4, xs + r * kXS);
        }
        __syncwarp();
        float y[2][4];
        forward16(ws, xs, r0, acts, y, lane);
        // relative L2 gradient at the output (columns 0..2 carry RGB)
        {
            const int rr = lane >> 2, q = lane & 3;
            float g[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t gi = base + r0 + rr + 8 * h;
                if (gi >= hi) continue;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = 2 * q + e;
                    if (c >= 3) continue;
                    const float yv = y[0][2 * h + e];
                    const float t = samples[4 * (size_t)gi + c].w;
                    const float den = yv * yv + kLossEps;
                    const float d = yv - t;
                    loss_sum += d * d / den;
                    g[h][e] = 2.0f * d / den * inv_batch;
                }
            }
            const int c = 2 * q;
            *reinterpret_cast<uint32_t*>(dz4 + (r0 + rr) * kZS + c) = pack_bf16(g[0][0], g[0][1]);
            *reinterpret_cast<uint32_t*>(dz4 + (r0 + rr + 8) * kZS + c) = pack_bf16(g[1][0], g[1][1]);
            *reinterpret_cast<uint32_t*>(dz4 + (r0 + rr) * kZS + 8 + c) = 0u;
            *reinterpret_cast<uint32_t*>(dz4 + (r0 + rr + 8) * kZS + 8 + c) = 0u;
        }
        __syncthreads();
        dw_layer<kU4>(acts[3], kAS, dz4, kZS, kOut / 8, g4, warp, lane);
        back16<kOut>(dz4, kZS, ws + w_smem_off(4), w_stride(4), acts[3], dz[1], r0, lane);
        __syncthreads();
        dw_layer<kU1>(acts[2], kAS, dz[1], kAS, kHid / 8, g3, warp, lane);
        back16<kHid>(dz[1], kAS, ws + w_smem_off(3), w_stride(3), acts[2], dz[0], r0, lane);
        __syncthreads();
        dw_layer<kU1>(acts[1], kAS, dz[0], kAS, kHid / 8, g2, warp, lane);
        back16<kHid>(dz[0], kAS, ws + w_smem_off(2), w_stride(2), acts[1], dz[1], r0, lane);
        __syncthreads();
        dw_layer<kU1>(acts[0], kAS, dz[1], kAS, kHid / 8, g1, warp, lane);
        back16<kHid>(dz[1], kAS, ws + w_smem_off(1), w_stride(1), acts[0], dz[0], r0, lane);
        __syncthreads();
        dw_layer<kU0>(xs, kXS, dz[0], kAS, kHid / 8, g0, warp, lane);
    }
    float* p = partials + (size_t)blockIdx.x * kParams;
    write_units<kU4>(p, 4, g4, warp, lane);
    write_units<kU1>(p, 3, g3, warp, lane);
    write_units<kU1>(p, 2, g2, warp, lane);
    write_units<kU1>(p, 1, g1, warp, lane);
    write_units<kU0>(p, 0, g0, warp, lane);
    if (loss) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) loss_sum += __shfl_xor_sync(0xFFFFFFFFu, loss_sum, o);
        if (lane == 0 && loss_sum != 0.f) atomicAdd(loss, loss_sum);
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(loss + 1, (float)batch);
    }
}

struct AdamArgs {
    float lr, beta1, beta2, eps, ema;
    float bc1, bc2, bce;  // 1 - beta1^t, 1 - beta2^t, 1 - ema^t
    int parts;
    uint32_t count_host, step, steps;
    const uint32_t* count_dev;
};

__global__ void __launch_bounds__(256) k_rc_adam(const float* __restrict__ partials, float* __restrict__ master,
                                                 float* __restrict__ m1, float* __restrict__ m2,
                                                 float* __restrict__ ema, bf16* __restrict__ w_train,
                                                 bf16* __restrict__ w_infer, AdamArgs a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    uint32_t lo, hi;
    batch_range(a.count_dev, a.count_host, a.step, a.steps, lo, hi);
    if (hi == lo) return;  // empty batch: no step
    float g = 0.f;
    for (int p = 0; p < a.parts; ++p) g += partials[(size_t)p * kParams + i];
    const float m = a.beta1 * m1[i] + (1.0f - a.beta1) * g;
    const float v = a.beta2 * m2[i] + (1.0f - a.beta2) * g * g;
    m1[i] = m;
    m2[i] = v;
    const float wv = master[i] - a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
    master[i] = wv;
    w_train[i] = __float2bfloat16_rn(wv);
    if (a.ema > 0.f) {
        const float e = a.ema * ema[i] + (1.0f - a.ema) * wv;
        ema[i] = e;
        w_infer[i] = __float2bfloat16_rn(e / a.bce);
    } else {
        w_infer[i] = __float2bfloat16_rn(wv);
    }
}

__global__ void k_rc_to_bf16(const float* __restrict__ master, bf16* __restrict__ w_train, bf16* __restrict__ w_infer,
                             float* __restrict__ ema)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    const bf16 b = __float2bfloat16_rn(master[i]);
    w_train[i] = b;
    w_infer[i] = b;
    ema[i] = 0.f;
}

// Training targets from the records of a finished wave: T = (R - R1) / W1 per
// channel (0 where W1 is 0: such a channel never uses the cache), clamped at 0.
// record_cap: records the buffer holds (appends past it were dropped).
__global__ void __launch_bounds__(256) k_rc_collect(const float4* __restrict__ records,
                                                    const uint32_t* __restrict__ record_count, uint32_t record_cap,
                                                    const float4* __restrict__ state, float4* __restrict__ samples,
                                                    uint32_t* __restrict__ sample_count, uint32_t capacity)
{
    const uint32_t n = min(*record_count, record_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 r0 = records[5 * (size_t)i], r1 = records[5 * (size_t)i + 1];
        const float4 r2 = records[5 * (size_t)i + 2], r3 = records[5 * (size_t)i + 3];
        const float4 r4 = records[5 * (size_t)i + 4];
        const float4 acc = state[2 * (size_t)__float_as_uint(r0.w)];
        const float tx = r1.w > 0.f ? fmaxf((acc.x - r4.x) / r1.w, 0.f) : 0.f;
        const float ty = r2.w > 0.f ? fmaxf((acc.y - r4.y) / r2.w, 0.f) : 0.f;
        const float tz = r3.w > 0.f ? fmaxf((acc.z - r4.z) / r3.w, 0.f) : 0.f;
        const uint32_t slot = atomicAdd(sample_count, 1u);
        if (slot >= capacity) continue;
        samples[4 * (size_t)slot] = make_float4(r0.x, r0.y, r0.z, tx);
        samples[4 * (size_t)slot + 1] = make_float4(r1.x, r1.y, r1.z, ty);
        samples[4 * (size_t)slot + 2] = make_float4(r2.x, r2.y, r2.z, tz);
        samples[4 * (size_t)slot + 3] = make_float4(r3.x, r3.y, r3.z, 0.f);
    }
}

// Kaiming-uniform initialisation from the Philox stream (key = seed, counter = index).
__global__ void k_rc_init(float* __restrict__ master, uint32_t seed)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kParams) return;
    int l = 0;
#pragma unroll
    for (int k = 1; k < kLayers; ++k)
        if (i >= param_off(k)) l = k;
    const float bound = sqrtf(6.0f / (float)fan_in(l)) * (l == kLayers - 1 ? 0.1f : 1.0f);
    const uint4 r = philox4x32_10(make_uint4((uint32_t)i, 0u, 0u, 0x52434E4Eu), seed, 0x9E3779B9u);
    master[i] = (2.0f * u01(r.x) - 1.0f) * bound;
}

}  // namespace rc
}  // namespace cpt

using namespace cpt;
using namespace cpt::rc;

struct cpt_rc {
    cpt_rc_params params{};
    int device = 0;
    float* master = nullptr;  // FP32 weights, [in][out] per layer, packed
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* ema = nullptr;
    bf16* w_train = nullptr;
    bf16* w_infer = nullptr;
    float* partials = nullptr;
    int parts = 0;
    float* loss = nullptr;      // [2] per cpt_rc_train call
    float* box = nullptr;       // [6] normalisation box for host-supplied boxes
    float4* samples = nullptr;  // training samples of the current frame
    uint32_t* sample_count = nullptr;
    uint32_t sample_cap = 0;
    float4* train_records = nullptr;  // vertex-1 records of the image's training paths (one wave)
    uint32_t* train_count = nullptr;
    uint32_t train_cap = 0;
    uint32_t t = 0;  // Adam steps taken
    void* block = nullptr;
};

namespace {

int train_grid()
{
    return std::min(kMaxTrainBlocks, sm_count());
}

bool g_attr_done[64];
std::mutex g_attr_mu;

int set_attributes()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CPT_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_attr_mu);
    if (g_attr_done[dev]) return CPT_OK;
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_rc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_rc_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_rc_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
    g_attr_done[dev] = true;
    return CPT_OK;
}

int infer_grid()
{
    static int occ = 0;
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_rc_infer<true>, kInferBlock, kInferSmem) !=
                cudaSuccess || occ < 1)
            occ = 1;
    }
    return sm_count() * occ;
}

// One training batch (step `step` of `steps` over the sample set) + Adam.
int train_batch(cpt_rc* rc, const float4* samples, const uint32_t* count_dev, uint32_t count_host, uint32_t step,
                uint32_t steps, const float* box, float* loss, cudaStream_t stream)
{
    {
        CPT_PROF(K_RC_TRAIN, stream);
        k_rc_train<<<rc->parts, kTrainBlock, kTrainSmem, stream>>>(rc->w_train, samples, count_dev, count_host, step,
                                                                   steps, box, rc->partials, loss);
    }
    CPT_LAUNCH_CHECK();
    rc->t += 1;
    AdamArgs a;
    a.lr = rc->params.learning_rate;
    a.beta1 = rc->params.beta1;
    a.beta2 = rc->params.beta2;
    a.eps = rc->params.epsilon;
    a.ema = rc->params.ema_decay;
    a.bc1 = 1.0f - powf(a.beta1, (float)rc->t);
    a.bc2 = 1.0f - powf(a.beta2, (float)rc->t);
    a.bce = a.ema > 0.f ? 1.0f - powf(a.ema, (float)rc->t) : 1.0f;
    a.parts = rc->parts;
    a.count_host = count_host;
    a.count_dev = count_dev;
    a.step = step;
    a.steps = steps;
    {
        CPT_PROF(K_RC_ADAM, stream);
        k_rc_adam<<<(kParams + 255) / 256, 256, 0, stream>>>(rc->partials, rc->master, rc->m1, rc->m2, rc->ema,
                                                             rc->w_train, rc->w_infer, a);
    }
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

struct Ctx {
    cpt_rc* rc;
    const float* box;
    bool training;    // a training-only pass: every record is a training record
    bool own_paths;   // an image pass with training paths among its own paths
};

int after_wave(void* ctx, const float4* records, const uint32_t* record_count, uint32_t capacity, float4* state,
               cudaStream_t stream)
{
    Ctx* c = static_cast<Ctx*>(ctx);
    if (c->training) {
        CPT_PROF(K_RC_COLLECT, stream);
        k_rc_collect<<<sm_count() * 4, 256, 0, stream>>>(records, record_count, capacity, state, c->rc->samples,
                                                         c->rc->sample_count, c->rc->sample_cap);
        CPT_LAUNCH_CHECK();
        return CPT_OK;
    }
    if (c->own_paths) {  // targets of this wave's training paths (their radiance is final now)
        {
            CPT_PROF(K_RC_COLLECT, stream);
            k_rc_collect<<<sm_count() * 4, 256, 0, stream>>>(c->rc->train_records, c->rc->train_count,
                                                             c->rc->train_cap, state, c->rc->samples,
                                                             c->rc->sample_count, c->rc->sample_cap);
        }
        CPT_LAUNCH_CHECK();
        CPT_CUDA_TRY(cudaMemsetAsync(c->rc->train_count, 0, sizeof(uint32_t), stream));  // the next wave's list
    }
    {
        CPT_PROF(K_RC_INFER, stream);
        k_rc_infer<true><<<infer_grid(), kInferBlock, kInferSmem, stream>>>(c->rc->w_infer, records, record_count, 0,
                                                                          c->box, state);
    }
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

// Per-view training resolution: about train_samples / n_views pixels with the
// view's aspect ratio.
void train_size(const cpt_view& v, uint32_t per_view, uint32_t& w, uint32_t& h)
{
    const double aspect = (double)v.width / (double)v.height;
    w = (uint32_t)std::max(1.0, floor(sqrt((double)per_view * aspect)));
    w = std::min(w, v.width);
    h = std::max(1u, std::min(v.height, per_view / w));
}

}  // namespace

extern "C" void cpt_rc_default_params(cpt_rc_params* p)
{
    if (!p) return;
    p->learning_rate = 1e-2f;
    p->beta1 = 0.9f;
    p->beta2 = 0.99f;
    p->epsilon = 1e-15f;
    p->ema_decay = 0.0f;
    p->train_samples = 1u << 16;
    p->train_steps = 4;
    p->seed = 1337u;
    p->train_interval = 1;
}

extern "C" size_t cpt_rc_param_count(void) { return (size_t)kParams; }

extern "C" int cpt_rc_create(cpt_rc** out, const cpt_rc_params* params, cudaStream_t stream)
{
    if (!out) return CPT_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cpt_rc_params p;
    cpt_rc_default_params(&p);
    if (params) p = *params;
    if (p.train_steps == 0 || p.train_samples == 0 || p.train_samples > (1u << 26) || !(p.learning_rate >= 0.f))
        return CPT_ERR_INVALID_ARGUMENT;
    int rc_ = set_attributes();
    if (rc_) return rc_;
    cpt_rc* rc = new (std::nothrow) cpt_rc();
    if (!rc) return CPT_ERR_CUDA;
    rc->params = p;
    cudaGetDevice(&rc->device);
    rc->parts = train_grid();
    rc->sample_cap = p.train_samples;
    Carver c(nullptr);
    c.take<float>(kParams);
    c.take<float>(kParams);
    c.take<float>(kParams);
    c.take<float>(kParams);
    c.take<bf16>(kParams);
    c.take<bf16>(kParams);
    c.take<float>((size_t)rc->parts * kParams);
    c.take<float>(2);
    c.take<float>(6);
    c.take<float4>(4ull * rc->sample_cap);
    c.take<uint32_t>(1);
    rc->train_cap = p.train_samples;
    c.take<float4>(5ull * rc->train_cap);
    c.take<uint32_t>(1);
    if (cudaMalloc(&rc->block, c.used()) != cudaSuccess) {
        delete rc;
        return CPT_ERR_CUDA;
    }
    Carver d(rc->block);
    rc->master = d.take<float>(kParams);
    rc->m1 = d.take<float>(kParams);
    rc->m2 = d.take<float>(kParams);
    rc->ema = d.take<float>(kParams);
    rc->w_train = d.take<bf16>(kParams);
    rc->w_infer = d.take<bf16>(kParams);
    rc->partials = d.take<float>((size_t)rc->parts * kParams);
    rc->loss = d.take<float>(2);
    rc->box = d.take<float>(6);
    rc->samples = d.take<float4>(4ull * rc->sample_cap);
    rc->sample_count = d.take<uint32_t>(1);
    rc->train_records = d.take<float4>(5ull * rc->train_cap);
    rc->train_count = d.take<uint32_t>(1);
    const int r = cpt_rc_reset(rc, p.seed, stream);
    if (r) {
        cpt_rc_destroy(rc);
        return r;
    }
    *out = rc;
    return CPT_OK;
}

extern "C" void cpt_rc_destroy(cpt_rc* rc)
{
    if (!rc) return;
    cudaDeviceSynchronize();
    if (rc->block) cudaFree(rc->block);
    delete rc;
}

extern "C" int cpt_rc_reset(cpt_rc* rc, uint32_t seed, cudaStream_t stream)
{
    if (!rc) return CPT_ERR_INVALID_ARGUMENT;
    rc->t = 0;
    CPT_CUDA_TRY(cudaMemsetAsync(rc->m1, 0, sizeof(float) * kParams, stream));
    CPT_CUDA_TRY(cudaMemsetAsync(rc->m2, 0, sizeof(float) * kParams, stream));
    k_rc_init<<<(kParams + 255) / 256, 256, 0, stream>>>(rc->master, seed);
    CPT_LAUNCH_CHECK();
    k_rc_to_bf16<<<(kParams + 255) / 256, 256, 0, stream>>>(rc->master, rc->w_train, rc->w_infer, rc->ema);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

extern "C" int cpt_rc_get_weights(cpt_rc* rc, float* host_out, cudaStream_t stream)
{
    if (!rc || !host_out) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(host_out, rc->master, sizeof(float) * kParams, cudaMemcpyDeviceToHost, stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    return CPT_OK;
}

extern "C" int cpt_rc_set_weights(cpt_rc* rc, const float* host_in, cudaStream_t stream)
{
    if (!rc || !host_in) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(rc->master, host_in, sizeof(float) * kParams, cudaMemcpyHostToDevice, stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    k_rc_to_bf16<<<(kParams + 255) / 256, 256, 0, stream>>>(rc->master, rc->w_train, rc->w_infer, rc->ema);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

extern "C" int cpt_rc_infer(cpt_rc* rc, const float* samples, uint32_t n, const float box[6], float* out,
                            cudaStream_t stream)
{
    CPT_RANGE("cpt_rc_infer");
    if (!rc || !box || (n && (!samples || !out))) return CPT_ERR_INVALID_ARGUMENT;
    if (!n) return CPT_OK;
    CPT_CUDA_TRY(cudaMemcpyAsync(rc->box, box, 6 * sizeof(float), cudaMemcpyHostToDevice, stream));
    {
        CPT_PROF(K_RC_INFER, stream);
        const int grid = std::min<int>(infer_grid(), (int)((n + 16 * kInferWarps - 1) / (16 * kInferWarps)));
        k_rc_infer<false><<<grid, kInferBlock, kInferSmem, stream>>>(
            rc->w_infer, reinterpret_cast<const float4*>(samples), nullptr, n, rc->box, reinterpret_cast<float4*>(out));
    }
    CPT_LAUNCH_CHECK();
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));  // the host box may go away
    return CPT_OK;
}

extern "C" int cpt_rc_train(cpt_rc* rc, const float* samples, uint32_t n, const float box[6], uint32_t steps,
                            float* loss_out, cudaStream_t stream)
{
    CPT_RANGE("cpt_rc_train");
    if (!rc || !box || !samples || n == 0 || steps == 0) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(rc->box, box, 6 * sizeof(float), cudaMemcpyHostToDevice, stream));
    CPT_CUDA_TRY(cudaMemsetAsync(rc->loss, 0, 2 * sizeof(float), stream));
    for (uint32_t s = 0; s < steps; ++s) {
        const int r = train_batch(rc, reinterpret_cast<const float4*>(samples), nullptr, n, s, steps, rc->box, rc->loss,
                                  stream);
        if (r) return r;
    }
    float l[2] = {0.f, 0.f};
    CPT_CUDA_TRY(cudaMemcpyAsync(l, rc->loss, sizeof(l), cudaMemcpyDeviceToHost, stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    if (loss_out) *loss_out = l[1] > 0.f ? l[0] / (3.0f * l[1]) : 0.f;
    return CPT_OK;
}

extern "C" size_t cpt_rc_render_scratch_bytes(const cpt_rc* rc, const cpt_view* views, uint32_t n_views,
                                              const cpt_render_params* params)
{
    if (!rc || !views || n_views == 0 || n_views > CPT_MAX_VIEWS || !params) return 0;
    cpt_render_params one = *params;
    one.wave_lanes = 1;  // cached renders run as one lane (their records are per wave)
    params = &one;
    std::vector<cpt_view> tv(views, views + n_views);
    const uint32_t per_view = std::max(1u, rc->params.train_samples / n_views);
    for (auto& v : tv) train_size(v, per_view, v.width, v.height);
    cpt_render_params pt = *params, pr = *params;
    pt.spp = 1;
    const size_t a = cpt_render_views_scratch_bytes(tv.data(), n_views, &pt);
    const size_t b = cpt_render_views_scratch_bytes(views, n_views, &pr);
    if (!a || !b) return 0;
    uint32_t cap = 0;
    const size_t ra = render_hook_layout(tv.data(), n_views, &pt, nullptr, &cap);
    const size_t rb = render_hook_layout(views, n_views, &pr, nullptr, &cap);
    return std::max(a, b) + std::max(ra, rb);
}

namespace {

int rc_frame(cpt_rc* rc, const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* scratch,
             size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status, bool image, cudaStream_t stream)
{
    if (!rc || !views || n_views == 0 || n_views > CPT_MAX_VIEWS || !params || !scratch || !status)
        return CPT_ERR_INVALID_ARGUMENT;
    const size_t need = cpt_rc_render_scratch_bytes(rc, views, n_views, params);
    if (!need) return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < need) return CPT_ERR_SCRATCH_TOO_SMALL;
    cpt_render_params one = *params;
    one.wave_lanes = 1;  // as sized above
    params = &one;
    std::vector<cpt_view> tv(views, views + n_views);
    const uint32_t per_view = std::max(1u, rc->params.train_samples / n_views);
    for (auto& v : tv) train_size(v, per_view, v.width, v.height);
    cpt_render_params pt = *params;
    pt.spp = 1;
    pt.seed_hi ^= 0xA511E9B3u;  // the training-only paths' own random stream
    pt.ray_sort = 0;
    pt.trace_stats = 0;
    uint32_t cap_t = 0, cap_r = 0;
    const size_t rec_t = render_hook_layout(tv.data(), n_views, &pt, nullptr, &cap_t);
    const size_t rec_r = render_hook_layout(views, n_views, params, nullptr, &cap_r);
    const size_t render_part = need - std::max(rec_t, rec_r);
    float4* records = reinterpret_cast<float4*>(static_cast<char*>(scratch) + render_part);
    const float* box = reinterpret_cast<const float*>(views[0].bvh->node_boxes);
    const uint32_t steps = rc->params.train_steps;
    if (!image) {
        // training only (cpt_rc_update): full-depth paths over reduced copies of the views,
        // records at vertex 1, targets, optimiser steps
        if (params->bounces < 2) return CPT_OK;
        CPT_CUDA_TRY(cudaMemsetAsync(rc->sample_count, 0, sizeof(uint32_t), stream));
        Ctx ct{rc, box, true, false};
        RenderHook h{};
        h.records = records;
        h.capacity = cap_t;
        h.record_depth = 1;
        h.image_pass = false;
        h.after_wave = after_wave;
        h.ctx = &ct;
        int r = cpt_render_views_hooked(tv.data(), n_views, &pt, scratch, render_part, ray_counts, status, &h, stream);
        if (r) return r;
        for (uint32_t s = 0; s < steps; ++s) {
            r = train_batch(rc, rc->samples, rc->sample_count, 0, s, steps, box, nullptr, stream);
            if (r) return r;
        }
        return CPT_OK;
    }
    if (params->bounces < 2)  // nothing after vertex 1 to cache: plain paths
        return cpt_render_views_hooked(views, n_views, params, scratch, render_part, ray_counts, status, nullptr,
                                       stream);
    // The image, training on its own paths: about train_samples of the frame's paths
    // (chosen by a hash of pixel and sample) are traced to full depth — their vertex-1
    // records give the training targets, their full estimate goes into the image — and
    // every other path stops at vertex 1 and takes the cache's prediction for the rest.
    const uint32_t interval = std::max(1u, rc->params.train_interval);
    const bool train = (params->frame0 / std::max(1u, params->spp)) % interval == 0;
    CPT_CUDA_TRY(cudaMemsetAsync(rc->sample_count, 0, sizeof(uint32_t), stream));
    CPT_CUDA_TRY(cudaMemsetAsync(rc->train_count, 0, sizeof(uint32_t), stream));
    uint64_t pixels = 0;
    for (uint32_t i = 0; i < n_views; ++i) pixels += (uint64_t)views[i].width * views[i].height;
    const uint64_t paths = pixels * params->spp;
    Ctx cr{rc, box, false, train};
    RenderHook h{};
    h.records = records;
    h.capacity = cap_r;
    h.record_depth = 1;
    h.image_pass = true;
    h.after_wave = after_wave;
    h.ctx = &cr;
    h.train_records = rc->train_records;
    h.train_count = rc->train_count;
    h.train_capacity = rc->train_cap;
    h.train_stride = train ? (uint32_t)std::max<uint64_t>(1, paths / std::max(1u, rc->params.train_samples)) : 0u;
    h.cut_at_record = true;
    int r = cpt_render_views_hooked(views, n_views, params, scratch, render_part, ray_counts, status, &h, stream);
    if (r || !train) return r;
    // optimiser steps over this frame's targets (the next frame's predictions use them)
    for (uint32_t s = 0; s < steps; ++s) {
        r = train_batch(rc, rc->samples, rc->sample_count, 0, s, steps, box, nullptr, stream);
        if (r) return r;
    }
    return CPT_OK;
}

}  // namespace

extern "C" int cpt_rc_render(cpt_rc* rc, const cpt_view* views, uint32_t n_views, const cpt_render_params* params,
                             void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                             cudaStream_t stream)
{
    CPT_RANGE("cpt_rc_render");
    return rc_frame(rc, views, n_views, params, scratch, scratch_bytes, ray_counts, status, true, stream);
}

extern "C" int cpt_rc_update(cpt_rc* rc, const cpt_view* views, uint32_t n_views, const cpt_render_params* params,
                             void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                             cudaStream_t stream)
{
    CPT_RANGE("cpt_rc_update");
    return rc_frame(rc, views, n_views, params, scratch, scratch_bytes, ray_counts, status, false, stream);
}

extern "C" int cpt_rc_sample_count(cpt_rc* rc, uint32_t* out, cudaStream_t stream)
{
    if (!rc || !out) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(out, rc->sample_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(stream));
    return CPT_OK;
}

extern "C" int cpt_rc_samples(cpt_rc* rc, const float** samples_dev)
{
    if (!rc || !samples_dev) return CPT_ERR_INVALID_ARGUMENT;
    *samples_dev = reinterpret_cast<const float*>(rc->samples);
    return CPT_OK;
}
