// Wavefront path tracer for sm_100a (cpt_render, cpt_render_views, cpt_resolve).
//
// The reference traces each pixel's whole path in one megakernel thread
// (raytrace_kernel, cuda_path_tracer.cu:385-421, with blinnPhongShadingPathTrace
// :245-333). Here a wave of paths advances one vertex at a time:
//
//   k_generate    primary rays for every (view, sample, pixel) of the wave -> queue 0
//   k_extend      closest hit for every ray in queue b                      -> hits
//   k_shade       shading of vertex b, shadow rays inline (any-hit),
//                 next bounce direction                                      -> queue b+1
//                 with next-event estimation: one shadow ray toward a point
//                 on the emitters and its weighted emission                  -> shadow queue
//   k_occlude     any-hit for every shadow ray; unoccluded ones add their
//                 emission to the path's radiance                            -> path state
//   k_accumulate  per pixel, the wave's samples in sample order              -> accumulators
//
// A "view" is one image: a BVH, its shading records and lights, a camera, a
// resolution and an accumulator. One call renders up to CPT_MAX_VIEWS views —
// several cameras of one scene, or many scenes (the batched workload) — in the
// same waves: the view table travels as a kernel parameter (so a frame is a fixed
// sequence of launches that a CUDA graph can capture), every ray carries its view
// index, and the traversal reads that view's nodes. Each path's radiance is the
// reference's estimator evaluated in the same operation order (round-to-nearest
// intrinsics), with random numbers from the counter-based Philox stream by
// (pixel, sample, bounce, view), so a path's result does not depend on queue order,
// wave size or which other views share the call. Within a view, a sample walks
// 8-row bands column by column so that a warp's primary rays cover a 4x8 patch.
#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>
#include "cpt.h"
#include "cpt_internal.h"
#include "traverse.cuh"
#include "onesweep.cuh"
#include "render_hook.h"

namespace cpt {

#ifndef CPT_EXTEND_BLOCK
#define CPT_EXTEND_BLOCK 128
#endif
constexpr int kExtendBlock = CPT_EXTEND_BLOCK;
#ifndef CPT_EXTEND_STEPS
#define CPT_EXTEND_STEPS 1024
#endif
constexpr int kExtendSteps = CPT_EXTEND_STEPS;  // most node visits between two refills of a warp
constexpr int kShadeBlock = 128;
constexpr int kGenBlock = 256;
constexpr int kMaxDepth = 62;  // bounces + 1 queues; reference GUI allows 5 bounces (PathTracingSettings.h:27)
constexpr uint32_t kDefaultWavePaths = 1u << 25;

struct Camera {
    float eye[3];
    float dirs[4][3];
    float m[16];
    float jx, jy;
    uint32_t jitter;
};

struct View {
    const float4* nodes;
    const float4* wide_nodes;  // compressed wide tree (cpt_lbvh_wide), nullable
    const float4* wide_tris;
    uint32_t wide_cap;         // its node capacity
    const cpt_triangle* tris;  // Morton-sorted reference records (info_idx of a hit)
    const cpt_triangle_info* infos;
    const cpt_dir_light* lights;
    const cudaTextureObject_t* textures;
    const float4* emitters;  // emitter table (next-event estimation), nullable
    void* accum;
    uint32_t info_count, light_count, max_visits, texture_count;
    uint32_t width, height, pixels, ref_w, ref_h;
    uint32_t pixel_base;  // pixels of the views before this one
    Camera cam;
};

struct Views {
    View v[CPT_MAX_VIEWS];
    uint32_t n;
    uint32_t total_pixels;
};

// Per-wave constants. A wave holds image-samples s0 .. s0+spw-1 of every view;
// paths are laid out view by view: view v owns paths
// [pixel_base(v) * spw, (pixel_base(v) + pixels(v)) * spw), sample-major inside.
struct Wave {
    uint32_t s0, spw;
    uint32_t p0, p1;  // the paths of the wave this launch sequence generates (a lane's half, or all)
    uint32_t frame0;
    const uint32_t* frame_dev;  // nullable: added to frame0 on the device (CUDA-graph replays)
    uint32_t bounces;
    float intensity;
    uint32_t stratified;
    uint32_t k0, k1;
    float4* records;          // nullable: vertex records (RenderHook)
    uint32_t* record_count;
    uint32_t record_depth;
    float4* train_records;    // training paths' records (RenderHook::train_stride > 0)
    uint32_t* train_count;
    uint32_t train_capacity;
    uint32_t train_stride;
    uint32_t cut_at_record;   // paths other than training paths end at record_depth
};

// Training-path selection of a (pixel, global sample) pair: a fixed integer hash
// (multiply / xor-shift rounds), so the choice does not depend on the wave layout.
__device__ __forceinline__ bool training_path(uint32_t pixel, uint32_t frame, uint32_t stride)
{
    uint32_t h = pixel * 0x9E3779B1u ^ (frame + 0x7F4A7C15u) * 0x85EBCA77u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h % stride == 0u;
}

// Slot -> pixel: 8-row bands, column-major inside a band.
__device__ __forceinline__ void slot_to_pixel(uint32_t slot, uint32_t w, uint32_t h, uint32_t& x, uint32_t& y)
{
    uint32_t band = slot / (8u * w);
    uint32_t bh = min(8u, h - 8u * band);
    uint32_t j = slot - band * 8u * w;
    x = j / bh;
    y = 8u * band + (j - x * bh);
}

__device__ __forceinline__ uint32_t pixel_to_slot(uint32_t x, uint32_t y, uint32_t w, uint32_t h)
{
    uint32_t band = y >> 3;
    uint32_t bh = min(8u, h - 8u * band);
    return band * 8u * w + x * bh + (y - 8u * band);
}

__device__ __forceinline__ void mat_vec(const float* m, float v0, float v1, float v2, float v3, float r[4])
{
#pragma unroll
    for (int row = 0; row < 4; ++row) {
        float a = __fmul_rn(m[row], v0), b = __fmul_rn(m[4 + row], v1);
        float c = __fmul_rn(m[8 + row], v2), d = __fmul_rn(m[12 + row], v3);
        r[row] = __fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d);
    }
}

// Corner directions of one sample (PathTracingApp.cpp:217-242 with the jitter
// from the Philox camera stream).
__device__ __forceinline__ void corner_dirs(const Camera& cam, uint32_t k0, uint32_t k1, uint32_t frame, f3 out[4])
{
    if (!cam.jitter) {
#pragma unroll
        for (int c = 0; c < 4; ++c) out[c] = mk3(cam.dirs[c][0], cam.dirs[c][1], cam.dirs[c][2]);
        return;
    }
    uint4 r = philox4x32_10(make_uint4(0xFFFFFFFFu, frame, 0u, 1u), k0, k1);
    float u0 = u01(r.x), u1 = u01(r.y);
    float jx = __fmul_rn(__fsub_rn(__fmul_rn(2.0f, u0), 1.0f), cam.jx);
    float jy = __fmul_rn(__fsub_rn(__fmul_rn(2.0f, u1), 1.0f), cam.jy);
    const float cx[4] = {-1.f, 1.f, 1.f, -1.f}, cy[4] = {-1.f, -1.f, 1.f, 1.f};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float nx = __fsub_rn(cx[c], jx), ny = __fsub_rn(cy[c], jy);
        float ws[4], we[4];
        mat_vec(cam.m, nx, ny, -1.0f, 1.0f, ws);
        mat_vec(cam.m, nx, ny, 1.0f, 1.0f, we);
        f3 ps = mk3(__fdiv_rn(ws[0], ws[3]), __fdiv_rn(ws[1], ws[3]), __fdiv_rn(ws[2], ws[3]));
        f3 pe = mk3(__fdiv_rn(we[0], we[3]), __fdiv_rn(we[1], we[3]), __fdiv_rn(we[2], we[3]));
        out[c] = normalize(sub(pe, ps));
    }
}

// Coherence key of a queued ray: direction octant (3 bits) above a 27-bit Morton
// code of the origin quantized to 512 cells per axis of the scene's root box.
// Also the 4 digit histograms of the keys and zeroing of the sort's look-back.
constexpr int kRayKeyPasses = 4;

__device__ __forceinline__ uint32_t spread3_10(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void __launch_bounds__(256) k_ray_keys(const float4* __restrict__ queue, const uint32_t* __restrict__ count,
                                                  const cpt_bbox* __restrict__ root, uint32_t* __restrict__ keys,
                                                  uint32_t* __restrict__ hist, uint32_t* __restrict__ zero,
                                                  size_t zero_words)
{
    __shared__ uint32_t s_hist[kRayKeyPasses * kRadix];
    for (int i = threadIdx.x; i < kRayKeyPasses * kRadix; i += blockDim.x) s_hist[i] = 0;
    const size_t gtid = (size_t)blockIdx.x * blockDim.x + threadIdx.x, gsize = (size_t)gridDim.x * blockDim.x;
    for (size_t i = gtid; i < zero_words; i += gsize) zero[i] = 0;
    __syncthreads();
    const uint32_t n = *count;
    const cpt_bbox b = *root;
    float inv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float ext = b.max[a] - b.min[a];
        inv[a] = ext > 0.f ? 511.0f / ext : 0.f;
    }
    for (uint32_t i = (uint32_t)gtid; i < n; i += (uint32_t)gsize) {
        const float4 o = queue[2 * (size_t)i], d = queue[2 * (size_t)i + 1];
        const float oo[3] = {o.x, o.y, o.z};
        uint32_t q[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float c = (oo[a] - b.min[a]) * inv[a];
            q[a] = (uint32_t)fminf(fmaxf(c, 0.0f), 511.0f);
        }
        const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
        const uint32_t key = (oct << 27) | spread3_10(q[0]) | (spread3_10(q[1]) << 1) | (spread3_10(q[2]) << 2);
        keys[i] = key;
#pragma unroll
        for (int p = 0; p < kRayKeyPasses; ++p) atomicAdd(&s_hist[p * kRadix + ((key >> (8 * p)) & 0xFFu)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRayKeyPasses * kRadix; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

// View owning global path p (binary search on the pixel bases).
__device__ __forceinline__ uint32_t view_of_path(const Views& vs, uint32_t p, uint32_t spw)
{
    uint32_t lo = 0, hi = vs.n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (vs.v[mid].pixel_base * spw <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t view_of_pixel(const Views& vs, uint32_t g)
{
    uint32_t lo = 0, hi = vs.n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (vs.v[mid].pixel_base <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ uint32_t wave_frame0(const Wave& wv) { return wv.frame0 + (wv.frame_dev ? *wv.frame_dev : 0u); }

__global__ void __launch_bounds__(kGenBlock) k_generate(Wave wv, Views vs, float4* __restrict__ queue,
                                                        uint32_t* __restrict__ counts, float4* __restrict__ state)
{
    const uint32_t frame0 = wave_frame0(wv);
    for (uint32_t pid = wv.p0 + blockIdx.x * kGenBlock + threadIdx.x; pid < wv.p1; pid += gridDim.x * kGenBlock) {
        const uint32_t vi = view_of_path(vs, pid, wv.spw);
        const View& v = vs.v[vi];
        const uint32_t local = pid - v.pixel_base * wv.spw;
        const uint32_t sl = local / v.pixels, slot = local - sl * v.pixels;
        uint32_t x, y;
        slot_to_pixel(slot, v.width, v.height, x, y);
        const bool live = x < v.ref_w && y < v.ref_h;
        state[2 * (size_t)pid] = make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t q = warp_append(&counts[0], live);
        if (!live) continue;
        f3 c[4];
        corner_dirs(v.cam, wv.k0, wv.k1, frame0 + wv.s0 + sl, c);
        // raytrace_kernel (cuda_path_tracer.cu:404-407): bilerp with (x/W, y/H), not normalised.
        const float tx = __fdiv_rn(__uint2float_rn(x), __uint2float_rn(v.width));
        const float ty = __fdiv_rn(__uint2float_rn(y), __uint2float_rn(v.height));
        const f3 d = mix3(mix3(c[0], c[1], tx), mix3(c[3], c[2], tx), ty);
        queue[2 * (size_t)q] = make_float4(v.cam.eye[0], v.cam.eye[1], v.cam.eye[2], __uint_as_float(pid));
        queue[2 * (size_t)q + 1] = make_float4(d.x, d.y, d.z, __uint_as_float(vi));
    }
}

// kOneView: every ray traverses view 0's BVH (a single scene, e.g. several cameras of
// it); the node array is then a kernel-wide constant instead of a per-ray value.
#ifndef CPT_EXTEND_MIN_BLOCKS
#define CPT_EXTEND_MIN_BLOCKS (1024 / CPT_EXTEND_BLOCK)  // 32 warps per SM: 64 registers
#endif
// kWide: every view's wide tree (cpt_lbvh_wide) instead of its binary nodes.
static_assert(kWideSmemStack * 2 == kSmemStack, "wide and binary stacks share the shared-memory buffer");
template <bool kStats, bool kOneView, bool kWide>
__global__ void __launch_bounds__(kExtendBlock, CPT_EXTEND_MIN_BLOCKS) k_extend(Views vs, const float4* __restrict__ queue,
                                                         const uint32_t* __restrict__ count, float4* __restrict__ hits,
                                                         uint32_t* __restrict__ pool,
                                                         unsigned long long* __restrict__ ray_counts,
                                                         uint32_t* __restrict__ status, const uint32_t* __restrict__ order,
                                                         uint32_t refill)
{
    __shared__ __align__(16) uint32_t s_stack[kSmemStack * kExtendBlock];
    const uint32_t n = *count;
    bool overflow = false;
    uint32_t nn = 0, nt = 0;
    if constexpr (kWide) {
        const float4* wn0 = vs.v[0].wide_nodes;
        const float4* wt0 = vs.v[0].wide_tris;
        const uint32_t cap0 = vs.v[0].wide_cap;
        auto wide_of = [&](uint32_t vi, uint32_t& mv, const float4*& tr) -> const float4* {
            if (kOneView) {
                mv = cap0;
                tr = wt0;
                return wn0;
            }
            mv = vs.v[vi].wide_cap;
            tr = vs.v[vi].wide_tris;
            return vs.v[vi].wide_nodes;
        };
        persistent_trace_wide<false, kExtendBlock, kStats, kExtendSteps, false>(
            wide_of, queue, n, pool, reinterpret_cast<uint2*>(s_stack) + threadIdx.x, overflow, nn, nt, order,
            [&](uint32_t ray, const WideState& s) {
                hits[ray] = make_float4(s.best.t, s.best.u, s.best.v, __uint_as_float(s.best.tri));
            },
            refill);
        if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
        if (kStats && ray_counts) {
            warp_count_u64(ray_counts + 3, nn);
            warp_count_u64(ray_counts + 4, nt);
        }
        return;
    }
    // each ray's view (direction .w) selects the node array it traverses
    const float4* nodes0 = vs.v[0].nodes;
    const uint32_t visits0 = vs.v[0].max_visits;
    auto view_nodes = [&](uint32_t vi, uint32_t& max_visits) -> const float4* {
        if (kOneView) {
            max_visits = visits0;
            return nodes0;
        }
        max_visits = vs.v[vi].max_visits;
        return vs.v[vi].nodes;
    };
    persistent_trace_views<false, kExtendBlock, kStats, kExtendSteps>(view_nodes, queue, n, hits, pool,
                                                                      s_stack + threadIdx.x, overflow, nn, nt, order,
                                                                      nullptr, refill);
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
    if (kStats && ray_counts) {
        warp_count_u64(ray_counts + 3, nn);
        warp_count_u64(ray_counts + 4, nt);
    }
}

// blinnPhongBRDF (cuda_path_tracer.cu:36-50)
__device__ __forceinline__ f3 blinn_phong(f3 Id, f3 kd, f3 Is, f3 ks, f3 n, f3 lv, f3 h, float shininess)
{
    float df = gmax(dot(n, lv), 0.0f);
    f3 diffuse = muls(mul(Id, kd), df);
    float sf = powf(gmax(dot(n, h), 0.0f), shininess);
    f3 spec = mk3(0.f, 0.f, 0.f);
    if (shininess > 0.0f && df > 0.0f) spec = muls(mul(Is, ks), sf);
    return add(diffuse, spec);
}

// toHemisphere (math_util.h:56-67)
__device__ __forceinline__ f3 to_hemisphere(f3 v, f3 n)
{
    f3 x = fabsf(n.x) < FLT_EPSILON ? cross(n, mk3(1.0f, 0.0f, 0.0f)) : cross(n, mk3(0.0f, 1.0f, 0.0f));
    x = normalize(x);
    f3 y = normalize(cross(n, x));
    return add(add(muls(x, v.x), muls(y, v.y)), muls(n, v.z));
}

// computeL (LightAlgorithms.h:12-20). The reference traces a full closest hit and
// tests distance < FLT_MAX; the any-hit traversal visits nodes in the same order
// until its first recorded triangle, so the visibility it returns is the same.
template <int kBlock>
__device__ __forceinline__ f3 light_l(const View& v, f3 p, const cpt_dir_light& l, uint32_t* stack, bool& overflow)
{
    const f3 dir = mk3(l.direction[0], l.direction[1], l.direction[2]);
    const f3 o = sub(p, muls(dir, 1e-3f));
    const Hit h = traverse<true, kBlock>(v.nodes, o, neg(dir), stack, overflow, v.max_visits);
    if (h.t < FLT_MAX) return mk3(0.f, 0.f, 0.f);
    return muls(mk3(l.color[0], l.color[1], l.color[2]), l.intensity);
}

// extractInfo / unpackNormal (cuda_path_tracer.cu:85-138): albedo from the albedo
// texture at the interpolated uv (as stored, not normalised) or the normalised
// interpolated vertex colour; normal from the normal map (2 * texel - 1 in the
// interpolated tangent frame, normalised) or the normalised interpolated normal.
// A texture index past the view's texture table is treated as absent.
__device__ __forceinline__ void surface(const View& v, const cpt_triangle_info& in, float u, float w, f3& albedo,
                                        f3& normal)
{
    normal = normalize(bary(ld3(in.vertices[0].normal), ld3(in.vertices[1].normal), ld3(in.vertices[2].normal), u, w));
    const uint32_t ai = in.material.albedo_idx, ni = in.material.normal_map_idx;
    const bool tex_a = ai < v.texture_count, tex_n = ni < v.texture_count;
    if (!tex_a && !tex_n) {
        albedo = normalize(bary(ld3(in.vertices[0].color), ld3(in.vertices[1].color), ld3(in.vertices[2].color), u, w));
        return;
    }
    // computeUV (TriangleInfo.h:71-74)
    const float tw = __fsub_rn(__fsub_rn(1.0f, u), w);
    const float tu = __fadd_rn(__fadd_rn(__fmul_rn(in.vertices[0].uv[0], tw), __fmul_rn(in.vertices[1].uv[0], u)),
                               __fmul_rn(in.vertices[2].uv[0], w));
    const float tv = __fadd_rn(__fadd_rn(__fmul_rn(in.vertices[0].uv[1], tw), __fmul_rn(in.vertices[1].uv[1], u)),
                               __fmul_rn(in.vertices[2].uv[1], w));
    if (tex_a) {
        const float4 c = tex2D<float4>(v.textures[ai], tu, tv);
        albedo = mk3(c.x, c.y, c.z);
    } else {
        albedo = normalize(bary(ld3(in.vertices[0].color), ld3(in.vertices[1].color), ld3(in.vertices[2].color), u, w));
    }
    if (tex_n) {
        const float4 ns = tex2D<float4>(v.textures[ni], tu, tv);
        const float nx = __fsub_rn(__fmul_rn(2.0f, ns.x), 1.0f), ny = __fsub_rn(__fmul_rn(2.0f, ns.y), 1.0f);
        const float nz = __fsub_rn(__fmul_rn(2.0f, ns.z), 1.0f);
        const f3 tg = normalize(bary(ld3(in.vertices[0].tangent), ld3(in.vertices[1].tangent), ld3(in.vertices[2].tangent), u, w));
        const f3 bt = normalize(bary(ld3(in.vertices[0].bitangent), ld3(in.vertices[1].bitangent),
                                     ld3(in.vertices[2].bitangent), u, w));
        normal = normalize(add(add(muls(tg, nx), muls(bt, ny)), muls(normal, nz)));
    }
}

constexpr uint32_t kNeeCounter = 0x10000u;  // Philox counter word 2 of the emitter draws: this + depth
constexpr float kPi = 3.14159265358979f;

// Next-event estimate at a vertex that bounces (position hp, shading normal n, ray
// origin of its bounce no = hp + n * 1e-5, path weight absorbed). The bounce it
// stands beside samples w with density max(n . w, 0) / pi and, where it hits an
// emitter, adds intensity * absorbed * e * max(-w . n_e, 0) (cuda_path_tracer.cu:
// 269-284, 303-312). Here a point y is drawn on the emitters with density 1 / A
// (a triangle by area, then uniformly on it), and the same integral over the
// emitters' area is estimated as
//     intensity * absorbed * e * max(-w . n_e, 0) * (n . w / pi) * |n_g . w| / r^2 * A,
// w = (y - no) / r, n_e the emitter's shading normal at y (the reference's
// `normal` of that hit), n_g its geometric normal. Returns false when the estimate
// is zero; otherwise the shadow ray (origin no, far limit 0.9999 r, direction w)
// and the emission it carries when unoccluded.
__device__ __forceinline__ bool nee_sample(const View& v, f3 no, f3 n, f3 absorbed, float intensity, uint32_t pixel,
                                           uint32_t frame, uint32_t depth, uint32_t vi, uint32_t k0, uint32_t k1,
                                           float4& ro, float4& rd, f3& c, bool& bad)
{
    const float4 hdr = __ldg(v.emitters);
    const uint32_t count = __float_as_uint(hdr.x);
    const float total = hdr.y;
    if (__float_as_uint(hdr.w)) bad = true;  // the table overflowed
    if (count == 0 || !(total > 0.0f)) return false;
    const uint4 r = philox4x32_10(make_uint4(pixel, frame, kNeeCounter + depth, vi), k0, k1);
    const float up = u01(r.x), s1 = u01(r.y), s2 = u01(r.z);
    const float4* rec = v.emitters + 1;
    uint32_t lo = 0, hi = count - 1;  // the first emitter with up < cdf
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (up < __ldg(&rec[3 * (size_t)mid].w)) hi = mid;
        else lo = mid + 1;
    }
    const float4 a = __ldg(rec + 3 * (size_t)lo), b = __ldg(rec + 3 * (size_t)lo + 1), e = __ldg(rec + 3 * (size_t)lo + 2);
    const f3 v0 = xyz(a), e1 = xyz(b), e2 = xyz(e);
    const float sq = __fsqrt_rn(s1);
    const float bu = __fmul_rn(sq, __fsub_rn(1.0f, s2)), bw = __fmul_rn(sq, s2);
    const f3 y = add(add(v0, muls(e1, bu)), muls(e2, bw));
    const f3 dv = sub(y, no);
    const float r2 = dot(dv, dv);
    if (!(r2 > 0.0f)) return false;
    const float dist = __fsqrt_rn(r2);
    const f3 w = muls(dv, __frcp_rn(dist));
    const float cos_x = dot(n, w);
    if (!(cos_x > 0.0f)) return false;
    const uint32_t tri = __float_as_uint(e.w);
    const uint32_t info_idx = __ldg(&v.tris[tri].info_idx);
    if (info_idx >= v.info_count) { bad = true; return false; }
    const cpt_triangle_info& in = v.infos[info_idx];
    f3 albedo_e, n_e;
    surface(v, in, bu, bw, albedo_e, n_e);
    const float cos_e = gmax(dot(neg(w), n_e), 0.0f);
    if (!(cos_e > 0.0f)) return false;
    const float cos_g = fabsf(dot(normalize(cross(e1, e2)), w));
    const float g = __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(cos_x, cos_e), cos_g), total), __fmul_rn(r2, kPi));
    c = muls(mul(absorbed, ld3(in.material.emission)), __fmul_rn(g, intensity));
    ro = make_float4(no.x, no.y, no.z, __fmul_rn(dist, 0.9999f));
    rd = make_float4(w.x, w.y, w.z, __uint_as_float(vi));
    return true;
}

// kNee: next-event estimation (cpt_render_params.nee): emission hit by a bounce ray
// is left out, and every vertex that bounces queues one shadow ray toward the
// emitters (nee_sample) for k_occlude.
template <bool kLights, bool kRecord, bool kNee>
__global__ void __launch_bounds__(kShadeBlock) k_shade(Views vs, Wave wv, uint32_t depth,
                                                       const float4* __restrict__ queue_in,
                                                       const float4* __restrict__ hits,
                                                       const uint32_t* __restrict__ count_in,
                                                       float4* __restrict__ queue_out, uint32_t* __restrict__ count_out,
                                                       float4* __restrict__ state,
                                                       unsigned long long* __restrict__ ray_counts,
                                                       uint32_t* __restrict__ status,
                                                       float4* __restrict__ shadow_rays,
                                                       float4* __restrict__ shadow_emission,
                                                       uint32_t* __restrict__ shadow_count)
{
    __shared__ uint32_t s_stack[kLights ? kSmemStack * kShadeBlock : 1];
    uint32_t* stack = s_stack + (kLights ? threadIdx.x : 0);
    const uint32_t n = *count_in;
    bool overflow = false;
    for (uint32_t base = blockIdx.x * kShadeBlock; base < n; base += gridDim.x * kShadeBlock) {
        const uint32_t i = base + threadIdx.x;
        bool emit = false;
        float4 nro = make_float4(0.f, 0.f, 0.f, 0.f), nrd = nro;
        uint32_t shadow = 0;
        bool bad_info = false;
        bool rec = false, train = false;
        float4 rec0, rec1, rec2, rec3, rec4;
        bool nee = false;
        float4 sro, srd;
        f3 sc;
        if (i < n) {
            const float4 ro = queue_in[2 * (size_t)i], rd4 = queue_in[2 * (size_t)i + 1];
            const float4 hit4 = hits[i];
            const uint32_t tri = __float_as_uint(hit4.w);
            const uint32_t pid = __float_as_uint(ro.w);
            const uint32_t vi = __float_as_uint(rd4.w);
            const View& v = vs.v[vi];
            const uint32_t info_idx = tri != CPT_INVALID_INDEX ? __ldg(&v.tris[tri].info_idx) : 0u;
            bad_info = tri != CPT_INVALID_INDEX && info_idx >= v.info_count;
            if (tri != CPT_INVALID_INDEX && !bad_info) {
                const f3 o = mk3(ro.x, ro.y, ro.z), d = mk3(rd4.x, rd4.y, rd4.z);
                const float t = hit4.x, u = hit4.y, w = hit4.z;
                const cpt_triangle_info& in = v.infos[info_idx];
                const f3 hp = add(muls(d, t), o);
                f3 albedo, normal;
                surface(v, in, u, w, albedo, normal);
                const f3 e = ld3(in.material.emission);
                const bool emissive = __fadd_rn(__fadd_rn(e.x, e.y), e.z) > 1e-7f;
                const float4 acc4 = state[2 * (size_t)pid], ab4 = state[2 * (size_t)pid + 1];
                f3 acc, absorbed;
                if (depth == 0) {
                    // blinnPhongShadingShadowTrace (cuda_path_tracer.cu:163-220)
                    if (emissive) {
                        albedo = mk3(1.f, 1.f, 1.f);
                        acc = e;
                    } else {
                        f3 L = mk3(0.f, 0.f, 0.f), color = mk3(0.f, 0.f, 0.f);
                        if (kLights) {
                            for (uint32_t li = 0; li < v.light_count; ++li) {
                                const cpt_dir_light l = v.lights[li];
                                L = add(L, light_l<kShadeBlock>(v, hp, l, stack, overflow));
                                ++shadow;
                                const f3 ldir = ld3(l.direction);
                                const f3 half = muls(sub(neg(d), ldir), 0.5f);
                                color = add(color, blinn_phong(L, albedo, L, mk3(0.5f, 0.5f, 0.5f), normal, neg(ldir), half,
                                                               in.material.specularity));
                            }
                        }
                        acc = color;
                    }
                    absorbed = albedo;
                } else {
                    // bounce vertex (cuda_path_tracer.cu:298-324)
                    acc = mk3(acc4.x, acc4.y, acc4.z);
                    absorbed = mk3(ab4.x, ab4.y, ab4.z);
                    f3 L = mk3(0.f, 0.f, 0.f);
                    if (emissive) {
                        if (!kNee) L = muls(e, gmax(dot(neg(d), normal), 0.0f));
                        albedo = mk3(1.f, 1.f, 1.f);
                    } else if (kLights) {
                        for (uint32_t li = 0; li < v.light_count; ++li) {
                            const cpt_dir_light l = v.lights[li];
                            const f3 c = light_l<kShadeBlock>(v, hp, l, stack, overflow);
                            ++shadow;
                            L = add(L, muls(c, gmax(dot(neg(ld3(l.direction)), normal), 0.0f)));
                        }
                    }
                    absorbed = mul(absorbed, albedo);
                    acc = add(acc, muls(mul(absorbed, L), wv.intensity));
                }
                state[2 * (size_t)pid] = make_float4(acc.x, acc.y, acc.z, 0.f);
                state[2 * (size_t)pid + 1] = make_float4(absorbed.x, absorbed.y, absorbed.z, 0.f);
                const uint32_t local = pid - v.pixel_base * wv.spw;
                const uint32_t sl = local / v.pixels, slot = local - sl * v.pixels;
                uint32_t x, y;
                slot_to_pixel(slot, v.width, v.height, x, y);
                const uint32_t frame = wave_frame0(wv) + wv.s0 + sl;
                bool go_on = depth < wv.bounces;
                if (kRecord && depth == wv.record_depth) {
                    rec = true;
                    rec0 = make_float4(hp.x, hp.y, hp.z, __uint_as_float(pid));
                    rec1 = make_float4(d.x, d.y, d.z, __fmul_rn(absorbed.x, wv.intensity));
                    rec2 = make_float4(normal.x, normal.y, normal.z, __fmul_rn(absorbed.y, wv.intensity));
                    rec3 = make_float4(albedo.x, albedo.y, albedo.z, __fmul_rn(absorbed.z, wv.intensity));
                    rec4 = make_float4(acc.x, acc.y, acc.z, 0.f);
                    train = wv.train_stride && training_path(v.pixel_base + y * v.width + x, frame, wv.train_stride);
                    if (train) rec = false;           // its record goes to the training list
                    else if (wv.cut_at_record) go_on = false;  // the cache supplies the rest
                }
                if (go_on) {
                    // next direction (cuda_path_tracer.cu:269-284)
                    const f3 no = add(hp, muls(normal, 1e-5f));
                    const uint4 r = philox4x32_10(make_uint4(y * v.width + x, frame, depth, vi), wv.k0, wv.k1);
                    float rx = u01(r.x), ry = u01(r.y);
                    if (wv.stratified && depth == 0) {
                        const uint32_t pos = frame % 64u;
                        rx = __fdiv_rn(__fadd_rn((float)(int)(pos % 8u), rx), 8.0f);
                        ry = __fdiv_rn(__fadd_rn((float)(int)(pos / 8u), ry), 8.0f);
                    }
                    float sn, cs;
                    sincos_turns(ry, &sn, &cs);
                    const float rr = __fsqrt_rn(rx);
                    const f3 dl = mk3(__fmul_rn(rr, cs), __fmul_rn(rr, sn), __fsqrt_rn(__fsub_rn(1.0f, rx)));
                    const f3 nd = to_hemisphere(dl, normal);
                    emit = true;
                    nro = make_float4(no.x, no.y, no.z, __uint_as_float(pid));
                    nrd = make_float4(nd.x, nd.y, nd.z, __uint_as_float(vi));
                    if (kNee)
                        nee = nee_sample(v, no, normal, absorbed, wv.intensity, y * v.width + x, frame, depth, vi,
                                         wv.k0, wv.k1, sro, srd, sc, bad_info);
                }
            }
        }
        const uint32_t q = warp_append(count_out, emit);
        if (emit) {
            queue_out[2 * (size_t)q] = nro;
            queue_out[2 * (size_t)q + 1] = nrd;
        }
        if (kRecord) {
            const uint32_t rq = warp_append(wv.record_count, rec);
            if (rec) {
                float4* r = wv.records + 5 * (size_t)rq;
                r[0] = rec0;
                r[1] = rec1;
                r[2] = rec2;
                r[3] = rec3;
                r[4] = rec4;
            }
            if (wv.train_stride) {
                const uint32_t tq = warp_append(wv.train_count, train);
                if (train && tq < wv.train_capacity) {
                    float4* r = wv.train_records + 5 * (size_t)tq;
                    r[0] = rec0;
                    r[1] = rec1;
                    r[2] = rec2;
                    r[3] = rec3;
                    r[4] = rec4;
                }
            }
        }
        if (kNee) {
            const uint32_t sq = warp_append(shadow_count, nee);
            if (nee) {
                shadow_rays[2 * (size_t)sq] = sro;
                shadow_rays[2 * (size_t)sq + 1] = srd;
                shadow_emission[sq] = make_float4(sc.x, sc.y, sc.z, __uint_as_float(__float_as_uint(nro.w)));
                ++shadow;
            }
        }
        if (kLights || kNee) warp_count_u64(ray_counts ? ray_counts + 2 : nullptr, shadow);
        if (bad_info) atomicOr(status, CPT_STATUS_BAD_INDEX);
    }
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
}

// Shadow rays of next-event estimation: any-hit up to each ray's far limit; an
// unoccluded ray adds its emission to its path's radiance (one shadow ray per
// path and vertex, so no two threads add to the same path).
template <bool kOneView, bool kWide>
__global__ void __launch_bounds__(kExtendBlock, CPT_EXTEND_MIN_BLOCKS) k_occlude(Views vs, const float4* __restrict__ rays,
                                                          const float4* __restrict__ emission,
                                                          const uint32_t* __restrict__ count,
                                                          uint32_t* __restrict__ pool, float4* __restrict__ state,
                                                          uint32_t* __restrict__ status)
{
    __shared__ __align__(16) uint32_t s_stack[kSmemStack * kExtendBlock];
    const uint32_t n = *count;
    bool overflow = false;
    uint32_t nn = 0, nt = 0;
    auto add_unoccluded = [&](uint32_t ray, const Hit& best) {
        if (best.tri != CPT_INVALID_INDEX) return;
        const float4 c = emission[ray];
        float4* st = state + 2 * (size_t)__float_as_uint(c.w);
        const float4 a = *st;
        *st = make_float4(__fadd_rn(a.x, c.x), __fadd_rn(a.y, c.y), __fadd_rn(a.z, c.z), a.w);
    };
    if constexpr (kWide) {
        auto wide_of = [&](uint32_t vi, uint32_t& mv, const float4*& tr) -> const float4* {
            const uint32_t v = kOneView ? 0u : vi;
            mv = vs.v[v].wide_cap;
            tr = vs.v[v].wide_tris;
            return vs.v[v].wide_nodes;
        };
        persistent_trace_wide<true, kExtendBlock, false, kExtendSteps, true>(
            wide_of, rays, n, pool, reinterpret_cast<uint2*>(s_stack) + threadIdx.x, overflow, nn, nt, nullptr,
            [&](uint32_t ray, const WideState& s) { add_unoccluded(ray, s.best); });
        if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
        return;
    }
    const float4* nodes0 = vs.v[0].nodes;
    const uint32_t visits0 = vs.v[0].max_visits;
    auto view_nodes = [&](uint32_t vi, uint32_t& max_visits) -> const float4* {
        if (kOneView) {
            max_visits = visits0;
            return nodes0;
        }
        max_visits = vs.v[vi].max_visits;
        return vs.v[vi].nodes;
    };
    persistent_trace<true, kExtendBlock, false, kExtendSteps, true>(
        view_nodes, rays, n, pool, s_stack + threadIdx.x, overflow, nn, nt, nullptr,
        [&](uint32_t ray, const TraceState& s) { add_unoccluded(ray, s.best); });
    if (overflow) atomicOr(status, CPT_STATUS_STACK_OVERFLOW);
}

// Primary / extension ray totals of a wave from the queue counters.
__global__ void k_wave_counts(const uint32_t* __restrict__ counts, uint32_t depth_count,
                              unsigned long long* __restrict__ ray_counts)
{
    if (threadIdx.x != 0 || !ray_counts) return;
    unsigned long long ext = 0;
    for (uint32_t b = 1; b < depth_count; ++b) ext += counts[b];
    atomicAdd(ray_counts + 0, (unsigned long long)counts[0]);
    atomicAdd(ray_counts + 1, ext);
    for (uint32_t b = 0; b < depth_count && b < 64; ++b) atomicAdd(ray_counts + 8 + b, (unsigned long long)counts[b]);
}

__global__ void k_advance(uint32_t* counter, uint32_t by) { *counter += by; }

// Adds the wave's samples to the accumulators, per pixel in sample order; one
// thread per pixel of every view.
__global__ void __launch_bounds__(256) k_accumulate(Wave wv, Views vs, uint32_t mode, const float4* __restrict__ state)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= vs.total_pixels) return;
    const View& v = vs.v[view_of_pixel(vs, g)];
    const uint32_t px = g - v.pixel_base;
    const uint32_t x = px % v.width, y = px / v.width;
    if (x >= v.ref_w || y >= v.ref_h) return;
    const uint32_t slot = pixel_to_slot(x, y, v.width, v.height);
    const size_t base = (size_t)v.pixel_base * wv.spw + slot;
    if (mode == CPT_ACCUM_KAHAN) {
        float4* sum = static_cast<float4*>(v.accum);
        float4* comp = sum + v.pixels;
        float4 s = sum[px], c = comp[px];
        for (uint32_t sl = 0; sl < wv.spw; ++sl) {
            const float4 r = state[2 * (base + (size_t)sl * v.pixels)];
            const float yx = __fsub_rn(r.x, c.x), yy = __fsub_rn(r.y, c.y), yz = __fsub_rn(r.z, c.z);
            const float tx = __fadd_rn(s.x, yx), ty = __fadd_rn(s.y, yy), tz = __fadd_rn(s.z, yz);
            c.x = __fsub_rn(__fsub_rn(tx, s.x), yx);
            c.y = __fsub_rn(__fsub_rn(ty, s.y), yy);
            c.z = __fsub_rn(__fsub_rn(tz, s.z), yz);
            s.x = tx; s.y = ty; s.z = tz;
            s.w = __fadd_rn(s.w, 1.0f);
        }
        sum[px] = s;
        comp[px] = c;
    } else if (mode == CPT_ACCUM_LERP) {
        // cuda_path_tracer.cu:413-420: new = lerp(hit, prev, f / (f + 1))
        float4* img = static_cast<float4*>(v.accum);
        const float4 p = img[px];
        f3 prev = mk3(p.x, p.y, p.z);
        for (uint32_t sl = 0; sl < wv.spw; ++sl) {
            const float4 r = state[2 * (base + (size_t)sl * v.pixels)];
            const float f = __uint2float_rn(wave_frame0(wv) + wv.s0 + sl);
            const float tt = __fdiv_rn(f, __fadd_rn(f, 1.0f));
            prev = mix3(mk3(r.x, r.y, r.z), prev, tt);
        }
        img[px] = make_float4(prev.x, prev.y, prev.z, 1.0f);
    } else {
        double4* sum = static_cast<double4*>(v.accum);
        double4 s = sum[px];
        for (uint32_t sl = 0; sl < wv.spw; ++sl) {
            const float4 r = state[2 * (base + (size_t)sl * v.pixels)];
            s.x += (double)r.x; s.y += (double)r.y; s.z += (double)r.z; s.w += 1.0;
        }
        sum[px] = s;
    }
}

__global__ void __launch_bounds__(256) k_resolve(const void* __restrict__ accum, uint32_t pixels, uint32_t mode,
                                                 float4* __restrict__ out)
{
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px >= pixels) return;
    if (mode == CPT_ACCUM_KAHAN) {
        float4 s = static_cast<const float4*>(accum)[px];
        float n = s.w;
        out[px] = n > 0.f ? make_float4(__fdiv_rn(s.x, n), __fdiv_rn(s.y, n), __fdiv_rn(s.z, n), 1.0f)
                          : make_float4(0.f, 0.f, 0.f, 1.0f);
    } else if (mode == CPT_ACCUM_LERP) {
        out[px] = static_cast<const float4*>(accum)[px];
    } else {
        double4 s = static_cast<const double4*>(accum)[px];
        out[px] = s.w > 0.0 ? make_float4((float)(s.x / s.w), (float)(s.y / s.w), (float)(s.z / s.w), 1.0f)
                            : make_float4(0.f, 0.f, 0.f, 1.0f);
    }
}

// Count words: queue counts, extension-ray pools, shadow-queue counts, shadow-ray
// pools (kMaxDepth + 2 each), then the record count.
constexpr int kCountWords = 4 * (kMaxDepth + 2) + 1;
constexpr int kShadowCountWord = 2 * (kMaxDepth + 2);
constexpr int kShadowPoolWord = 3 * (kMaxDepth + 2);
constexpr int kRecordCountWord = 4 * (kMaxDepth + 2);

// What one lane of a wave owns: its ray queues, hits, counters and shadow-ray queue
// (paths and their state belong to the wave).
struct Lane {
    float4* queue[2];
    float4* hits;
    uint32_t* counts;
    float4* shadow_rays;      // next-event estimation: 2 float4 per shadow ray
    float4* shadow_emission;  // and its emission | path id
};

struct RenderScratch {
    float4* queue[2];
    float4* hits;
    float4* state;
    uint32_t* counts;
    uint32_t capacity;  // paths per wave
    float4* shadow_rays;      // next-event estimation: 2 float4 per shadow ray
    float4* shadow_emission;  // and its emission | path id
    Lane second;              // the second lane (wave_lanes 2): queues for half the capacity
    bool two_lanes;
    // coherence sort of bounce queues
    uint32_t* sort_keys[2];
    uint32_t* sort_vals[2];
    uint32_t* sort_hist;
    uint32_t* sort_offsets;
    uint32_t* sort_zero;  // tile counters (32 words) + look-back
    size_t sort_zero_words;
};

// Lanes per wave the scratch is laid out for: 2 on request (not with ray sorting, whose
// buffers are the wave's), else 1. A call with a render hook uses one lane whatever the
// scratch holds. Measured (events per frame): C3's 64 views 1067 -> 1099 Mrays/s with
// two lanes; C2 516 -> 514 and C1 400 -> 369 (small waves pay for the second sequence
// of launches), so one lane is the default and the autotuner tries two.
inline uint32_t wave_lanes(const cpt_render_params* p)
{
    return (p->wave_lanes == 2 && !p->ray_sort) ? 2u : 1u;
}

// Image-samples per wave for `pixels` pixels over all views.
inline uint32_t wave_samples(const cpt_render_params* p, uint64_t pixels)
{
    const uint64_t want = p->wave_paths ? p->wave_paths : kDefaultWavePaths;
    uint64_t spw = want / pixels;
    if (spw < 1) spw = 1;
    if (spw > p->spp) spw = p->spp;
    return (uint32_t)spw;
}

size_t render_layout(const cpt_render_params* p, uint64_t pixels, void* base, RenderScratch* out)
{
    Carver c(base);
    RenderScratch s;
    s.capacity = (uint32_t)(pixels * wave_samples(p, pixels));
    s.queue[0] = c.take<float4>(2ull * s.capacity);
    s.queue[1] = c.take<float4>(2ull * s.capacity);
    s.hits = c.take<float4>(s.capacity);
    s.state = c.take<float4>(2ull * s.capacity);
    s.counts = c.take<uint32_t>(kCountWords);  // queue counts, persistent-kernel ray pools, record count
    if (p->nee) {
        s.shadow_rays = c.take<float4>(2ull * s.capacity);
        s.shadow_emission = c.take<float4>(s.capacity);
    } else {
        s.shadow_rays = s.shadow_emission = nullptr;
    }
    s.two_lanes = wave_lanes(p) == 2;
    if (s.two_lanes) {
        const uint64_t half = s.capacity / 2 + 1;
        s.second.queue[0] = c.take<float4>(2ull * half);
        s.second.queue[1] = c.take<float4>(2ull * half);
        s.second.hits = c.take<float4>(half);
        s.second.counts = c.take<uint32_t>(kCountWords);
        if (p->nee) {
            s.second.shadow_rays = c.take<float4>(2ull * half);
            s.second.shadow_emission = c.take<float4>(half);
        } else {
            s.second.shadow_rays = s.second.shadow_emission = nullptr;
        }
    } else {
        s.second = Lane{};
    }
    if (p->ray_sort) {
        const size_t tiles = (s.capacity + kSortTile - 1) / kSortTile;
        for (int k = 0; k < 2; ++k) {
            s.sort_keys[k] = c.take<uint32_t>(s.capacity);
            s.sort_vals[k] = c.take<uint32_t>(s.capacity);
        }
        s.sort_hist = c.take<uint32_t>(kRayKeyPasses * kRadix);
        s.sort_offsets = c.take<uint32_t>(kRayKeyPasses * kRadix);
        s.sort_zero_words = 32 + (size_t)kRayKeyPasses * tiles * kRadix;
        s.sort_zero = c.take<uint32_t>(s.sort_zero_words);
    } else {
        s.sort_keys[0] = s.sort_keys[1] = s.sort_vals[0] = s.sort_vals[1] = nullptr;
        s.sort_hist = s.sort_offsets = s.sort_zero = nullptr;
        s.sort_zero_words = 0;
    }
    if (out) *out = s;
    return c.used();
}

// Sorts the `*count` rays of `queue` by coherence key; the permutation ends in
// rs.sort_vals[(kRayKeyPasses - 1) & 1]. Grids are sized for the wave capacity;
// the kernels read the actual count on the device.
int sort_queue(const RenderScratch& rs, const float4* queue, const uint32_t* count, const cpt_bbox* root,
               uint32_t* status, cudaStream_t stream)
{
    const uint32_t tiles = (rs.capacity + kSortTile - 1) / kSortTile;
    const int sms = sm_count();
    CPT_CUDA_TRY(cudaMemsetAsync(rs.sort_hist, 0, sizeof(uint32_t) * kRayKeyPasses * kRadix, stream));
    {
        CPT_PROF(K_RAY_SORT, stream);
        k_ray_keys<<<sms * 8, 256, 0, stream>>>(queue, count, root, rs.sort_keys[0], rs.sort_hist, rs.sort_zero,
                                                rs.sort_zero_words);
    }
    CPT_LAUNCH_CHECK();
    {
        CPT_PROF(K_RAY_SORT, stream);
        k_scan_offsets<<<kRayKeyPasses, kRadix, 0, stream>>>(rs.sort_hist, rs.sort_offsets);
    }
    CPT_LAUNCH_CHECK();
    const size_t smem = onesweep_smem<uint32_t>();
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<uint32_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CPT_CUDA_TRY(cudaFuncSetAttribute(k_onesweep<uint32_t, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    uint32_t* lookback = rs.sort_zero + 32;
    for (int p = 0; p < kRayKeyPasses; ++p) {
        const uint32_t* kin = rs.sort_keys[p & 1];
        uint32_t* kout = rs.sort_keys[(p + 1) & 1];
        const uint32_t* vin = p == 0 ? nullptr : rs.sort_vals[(p + 1) & 1];
        uint32_t* vout = rs.sort_vals[p & 1];
        CPT_PROF(K_RAY_SORT, stream);
        if (p == 0)
            k_onesweep<uint32_t, true><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, 0, count, 8 * p,
                                                                            rs.sort_offsets + p * kRadix,
                                                                            lookback + (size_t)p * tiles * kRadix,
                                                                            rs.sort_zero + p, status);
        else
            k_onesweep<uint32_t, false><<<tiles, kSortBlock, smem, stream>>>(kin, vin, kout, vout, 0, count, 8 * p,
                                                                             rs.sort_offsets + p * kRadix,
                                                                             lookback + (size_t)p * tiles * kRadix,
                                                                             rs.sort_zero + p, status);
        CPT_LAUNCH_CHECK();
    }
    return CPT_OK;
}

bool params_ok(const cpt_render_params* p, uint64_t pixels)
{
    if (!p || p->spp == 0 || pixels == 0 || pixels > (1ull << 31)) return false;
    if (p->bounces + 1 > (uint32_t)kMaxDepth) return false;
    if (p->accum_mode > CPT_ACCUM_F64 || p->nee > 1 || p->wave_lanes > 2) return false;
    return pixels * wave_samples(p, pixels) < (1ull << 31);
}

inline uint32_t camera_count(const cpt_render_params* p) { return p->cameras ? p->cameras : 1u; }

void to_camera(const cpt_camera& src, Camera& cam)
{
    for (int a = 0; a < 3; ++a) cam.eye[a] = src.eye[a];
    for (int c = 0; c < 4; ++c)
        for (int a = 0; a < 3; ++a) cam.dirs[c][a] = src.dirs[c][a];
    for (int k = 0; k < 16; ++k) cam.m[k] = src.inv_view_proj[k];
    cam.jx = src.jitter_x;
    cam.jy = src.jitter_y;
    cam.jitter = src.jitter;
}

// Fills the kernel-parameter view table; returns total pixels or 0 on a bad view.
uint64_t make_views(const cpt_view* views, uint32_t n, uint32_t ref_grid, bool nee, Views& vs)
{
    uint64_t total = 0;
    vs.n = n;
    for (uint32_t i = 0; i < n; ++i) {
        const cpt_view& s = views[i];
        if (!s.bvh || !s.scene || !s.bvh->nodes || !s.bvh->tris || !s.scene->infos || !s.accum || s.width == 0 ||
            s.height == 0 || (s.scene->light_count && !s.scene->lights) || (reinterpret_cast<uintptr_t>(s.accum) & 15) ||
            (nee && (!s.scene->emitters || (reinterpret_cast<uintptr_t>(s.scene->emitters) & 15))))
            return 0;
        View& v = vs.v[i];
        v.nodes = static_cast<const float4*>(s.bvh->split_nodes ? s.bvh->split_nodes : s.bvh->nodes);
        v.wide_nodes = static_cast<const float4*>(s.bvh->wide_nodes);
        v.wide_tris = static_cast<const float4*>(s.bvh->wide_tris);
        v.wide_cap = s.bvh->wide_nodes ? s.bvh->wide_capacity - 1 : 0u;
        v.tris = s.bvh->tris;
        v.infos = s.scene->infos;
        v.lights = s.scene->lights;
        v.textures = s.scene->textures;
        v.emitters = nee ? static_cast<const float4*>(s.scene->emitters) : nullptr;
        v.texture_count = s.scene->textures ? s.scene->texture_count : 0u;
        v.accum = s.accum;
        v.info_count = s.scene->info_count;
        v.light_count = s.scene->light_count;
        // a ray fetches each internal node at most once
        v.max_visits = s.bvh->split_nodes ? (s.bvh->split_capacity | kFastSlabBit) : s.bvh->n;
        v.width = s.width;
        v.height = s.height;
        v.pixels = s.width * s.height;
        v.ref_w = ref_grid ? s.width / 8u * 8u : s.width;
        v.ref_h = ref_grid ? s.height / 8u * 8u : s.height;
        v.pixel_base = (uint32_t)total;
        to_camera(s.camera, v.cam);
        total += (uint64_t)s.width * s.height;
        if (total >= (1ull << 31)) return 0;
    }
    vs.total_pixels = (uint32_t)total;
    return total;
}

// The second lane's stream and the three events that order it against the caller's
// stream (fork at the wave's start, the one-launch stagger, the join before the
// accumulation), one set per device, created on first use and kept for the process.
struct LaneStreams {
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, stagger = nullptr, join = nullptr;
};
constexpr uint32_t kMinLanePaths = 1u << 12;  // waves below twice this run as one lane

LaneStreams* lane_streams()
{
    constexpr int kMaxDevices = 64;
    static LaneStreams table[kMaxDevices];
    static std::mutex mu;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    LaneStreams& l = table[dev];
    if (!l.stream) {
        cudaStream_t st = nullptr;
        cudaEvent_t e[3] = {nullptr, nullptr, nullptr};
        bool ok = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess;
        for (int k = 0; k < 3 && ok; ++k) ok = cudaEventCreateWithFlags(&e[k], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) {
            for (int k = 0; k < 3; ++k)
                if (e[k]) cudaEventDestroy(e[k]);
            if (st) cudaStreamDestroy(st);
            return nullptr;
        }
        l.fork = e[0];
        l.stagger = e[1];
        l.join = e[2];
        l.stream = st;
    }
    return &l;
}

int render_views(const Views& vs, bool any_lights, const cpt_bbox* sort_root, const cpt_render_params* params,
                 void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                 const RenderHook* hook, cudaStream_t stream)
{
    const uint64_t pixels = vs.total_pixels;
    if (!params_ok(params, pixels) || !scratch || !status) return CPT_ERR_INVALID_ARGUMENT;
    if (scratch_bytes < render_layout(params, pixels, nullptr, nullptr)) return CPT_ERR_SCRATCH_TOO_SMALL;
    if (reinterpret_cast<uintptr_t>(scratch) & 255) return CPT_ERR_INVALID_ARGUMENT;
    RenderScratch rs;
    render_layout(params, pixels, scratch, &rs);

    Wave wv;
    wv.frame0 = params->frame0;
    wv.frame_dev = params->frame_counter;
    wv.bounces = params->bounces;
    wv.intensity = params->indirect_intensity;
    wv.stratified = params->stratified;
    wv.k0 = params->seed_lo;
    wv.k1 = params->seed_hi;
    const bool record = hook && hook->records;
    if (record && hook->capacity < rs.capacity) return CPT_ERR_SCRATCH_TOO_SMALL;
    wv.records = record ? hook->records : nullptr;
    wv.record_count = rs.counts + kRecordCountWord;
    wv.record_depth = hook ? hook->record_depth : 0u;
    const bool train = record && hook->train_stride && hook->train_records && hook->train_count;
    wv.train_records = train ? hook->train_records : nullptr;
    wv.train_count = train ? hook->train_count : nullptr;
    wv.train_capacity = train ? hook->train_capacity : 0u;
    wv.train_stride = train ? hook->train_stride : 0u;
    wv.cut_at_record = record && hook->cut_at_record ? 1u : 0u;
    const bool image = !hook || hook->image_pass;

    bool one_bvh = true, wide = true;
    for (uint32_t i = 1; i < vs.n; ++i) one_bvh &= vs.v[i].nodes == vs.v[0].nodes;
    for (uint32_t i = 0; i < vs.n; ++i) wide &= vs.v[i].wide_nodes != nullptr;  // else every view's binary tree
    const int sms = sm_count();
    static int ext_occ = 0;
    if (!ext_occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ext_occ, k_extend<false, false, false>, kExtendBlock, 0) != cudaSuccess ||
            ext_occ < 1)
            ext_occ = 1;
    }
    // Two lanes: the wave's paths split in halves, the second half on the library's own
    // stream, its first traversal launch one launch behind the first half's, the halves
    // joined before the wave's accumulation (paths and their state are the wave's, so
    // the image is the one-lane image).
    const bool two = rs.two_lanes && !hook;
    LaneStreams* ls = nullptr;
    if (two) {
        ls = lane_streams();
        if (!ls) return CPT_ERR_CUDA;
    }
    const Lane first{{rs.queue[0], rs.queue[1]}, rs.hits, rs.counts, rs.shadow_rays, rs.shadow_emission};
    // launch shape of the persistent traversal: resident blocks per SM (occupancy, or the
    // caller's smaller figure) and the refill threshold of its warps (0: the default)
    const int per_sm = params->traverse_blocks_per_sm ? std::min<int>(ext_occ, (int)params->traverse_blocks_per_sm)
                                                      : ext_occ;
    const uint32_t refill = std::min<uint32_t>(params->refill_lanes, 32u);

    // Generation, every vertex's extension + shading (+ shadow rays), and the lane's ray
    // counts, for the wave's paths [wl.p0, wl.p1) on stream st. after_first (nullable):
    // recorded after the lane's first traversal launch; before_first (nullable): waited
    // on before it.
    auto run_lane = [&](const Lane& L, const Wave& wl, cudaStream_t st, cudaEvent_t after_first,
                        cudaEvent_t before_first) -> int {
        const uint32_t paths = wl.p1 - wl.p0;
        CPT_CUDA_TRY(cudaMemsetAsync(L.counts, 0, sizeof(uint32_t) * kCountWords, st));
        {
            CPT_PROF(K_GENERATE, st);
            k_generate<<<(int)std::min<uint32_t>((paths + kGenBlock - 1) / kGenBlock, (uint32_t)sms * 16), kGenBlock, 0,
                         st>>>(wl, vs, L.queue[0], L.counts, rs.state);
        }
        CPT_LAUNCH_CHECK();
        const int ext_blocks = std::min<int>((int)((paths + kExtendBlock - 1) / kExtendBlock), sms * per_sm);
        const int shade_blocks = std::min<int>((int)((paths + kShadeBlock - 1) / kShadeBlock), sms * 16);
        for (uint32_t b = 0; b <= params->bounces; ++b) {
            const float4* qin = L.queue[b & 1];
            float4* qout = L.queue[(b + 1) & 1];
            const uint32_t* order = nullptr;
            if (params->ray_sort && b > 0) {
                const int rc = sort_queue(rs, qin, L.counts + b, sort_root, status, st);
                if (rc != CPT_OK) return rc;
                order = rs.sort_vals[(kRayKeyPasses - 1) & 1];
            }
            if (b == 0 && before_first) CPT_CUDA_TRY(cudaStreamWaitEvent(st, before_first, 0));
            {
                CPT_PROF(K_EXTEND, st);
                uint32_t* pool = L.counts + kMaxDepth + 2 + b;
#define CPT_EXTEND(S, O, W) \
    k_extend<S, O, W><<<ext_blocks, kExtendBlock, 0, st>>>(vs, qin, L.counts + b, L.hits, pool, ray_counts, status, \
                                                           order, refill)
                if (wide) {
                    if (params->trace_stats) {
                        if (one_bvh) CPT_EXTEND(true, true, true); else CPT_EXTEND(true, false, true);
                    } else {
                        if (one_bvh) CPT_EXTEND(false, true, true); else CPT_EXTEND(false, false, true);
                    }
                } else if (params->trace_stats) {
                    if (one_bvh) CPT_EXTEND(true, true, false); else CPT_EXTEND(true, false, false);
                } else {
                    if (one_bvh) CPT_EXTEND(false, true, false); else CPT_EXTEND(false, false, false);
                }
#undef CPT_EXTEND
            }
            CPT_LAUNCH_CHECK();
            if (b == 0 && after_first) CPT_CUDA_TRY(cudaEventRecord(after_first, st));
            const bool nee_here = params->nee && b < params->bounces;
            if (hook && hook->shade_after && wl.s0 == 0 && b == 0)
                CPT_CUDA_TRY(cudaStreamWaitEvent(st, hook->shade_after, 0));
            {
                CPT_PROF(K_SHADE, st);
#define CPT_SHADE(LI, R, N)                                                                                         \
    k_shade<LI, R, N><<<shade_blocks, kShadeBlock, 0, st>>>(vs, wl, b, qin, L.hits, L.counts + b, qout,            \
                                                            L.counts + b + 1, rs.state, ray_counts, status,        \
                                                            L.shadow_rays, L.shadow_emission,                      \
                                                            L.counts + kShadowCountWord + b)
                const bool rec_here = record && b == wl.record_depth;
                if (params->nee) {  // (the last vertex queues no shadow ray: it does not bounce)
                    if (any_lights) {
                        if (rec_here) CPT_SHADE(true, true, true); else CPT_SHADE(true, false, true);
                    } else {
                        if (rec_here) CPT_SHADE(false, true, true); else CPT_SHADE(false, false, true);
                    }
                } else {
                    if (any_lights) {
                        if (rec_here) CPT_SHADE(true, true, false); else CPT_SHADE(true, false, false);
                    } else {
                        if (rec_here) CPT_SHADE(false, true, false); else CPT_SHADE(false, false, false);
                    }
                }
#undef CPT_SHADE
            }
            CPT_LAUNCH_CHECK();
            if (nee_here) {
                CPT_PROF(K_OCCLUDE, st);
                uint32_t* spool = L.counts + kShadowPoolWord + b;
                const uint32_t* scount = L.counts + kShadowCountWord + b;
#define CPT_OCCLUDE(O, W)                                                                                   \
    k_occlude<O, W><<<ext_blocks, kExtendBlock, 0, st>>>(vs, L.shadow_rays, L.shadow_emission, scount, spool, \
                                                         rs.state, status)
                if (wide) {
                    if (one_bvh) CPT_OCCLUDE(true, true); else CPT_OCCLUDE(false, true);
                } else {
                    if (one_bvh) CPT_OCCLUDE(true, false); else CPT_OCCLUDE(false, false);
                }
#undef CPT_OCCLUDE
                CPT_LAUNCH_CHECK();
            }
        }
        if (ray_counts) {
            {
                CPT_PROF(K_WAVE_COUNTS, st);
                k_wave_counts<<<1, 32, 0, st>>>(L.counts, params->bounces + 1, ray_counts);
            }
            CPT_LAUNCH_CHECK();
        }
        return CPT_OK;
    };

    const uint32_t spw_max = wave_samples(params, pixels);
    for (uint32_t s0 = 0; s0 < params->spp; s0 += spw_max) {
        wv.s0 = s0;
        wv.spw = std::min(spw_max, params->spp - s0);
        const uint32_t paths = wv.spw * vs.total_pixels;
        if (two && paths >= 2 * kMinLanePaths) {
            Wave wa = wv, wb = wv;
            wa.p0 = 0;
            wa.p1 = paths / 2;
            wb.p0 = paths / 2;
            wb.p1 = paths;
            CPT_CUDA_TRY(cudaEventRecord(ls->fork, stream));
            CPT_CUDA_TRY(cudaStreamWaitEvent(ls->stream, ls->fork, 0));
            if (const int rc = run_lane(first, wa, stream, ls->stagger, nullptr)) return rc;
            if (const int rc = run_lane(rs.second, wb, ls->stream, nullptr, ls->stagger)) return rc;
            CPT_CUDA_TRY(cudaEventRecord(ls->join, ls->stream));
            CPT_CUDA_TRY(cudaStreamWaitEvent(stream, ls->join, 0));
        } else {
            wv.p0 = 0;
            wv.p1 = paths;
            if (const int rc = run_lane(first, wv, stream, nullptr, nullptr)) return rc;
        }
        if (hook && hook->after_wave) {
            const int rc = hook->after_wave(hook->ctx, hook->records, wv.record_count, hook->capacity, rs.state, stream);
            if (rc != CPT_OK) return rc;
        }
        if (!image) continue;
        {
            CPT_PROF(K_ACCUMULATE, stream);
            k_accumulate<<<(vs.total_pixels + 255) / 256, 256, 0, stream>>>(wv, vs, params->accum_mode, rs.state);
        }
        CPT_LAUNCH_CHECK();
    }
    if (params->frame_counter && image) {
        k_advance<<<1, 1, 0, stream>>>(params->frame_counter, params->spp);
        CPT_LAUNCH_CHECK();
    }
    return CPT_OK;
}

}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_accum_bytes(uint32_t width, uint32_t height, uint32_t accum_mode)
{
    const size_t px = (size_t)width * height;
    if (accum_mode == CPT_ACCUM_KAHAN) return px * 2 * sizeof(float4);
    if (accum_mode == CPT_ACCUM_LERP) return px * sizeof(float4);
    if (accum_mode == CPT_ACCUM_F64) return px * sizeof(double4);
    return 0;
}

extern "C" size_t cpt_render_scratch_bytes(const cpt_render_params* params)
{
    if (!params || params->width == 0 || params->height == 0 || camera_count(params) > CPT_MAX_VIEWS) return 0;
    const uint64_t pixels = (uint64_t)params->width * params->height * camera_count(params);
    if (!params_ok(params, pixels)) return 0;
    return render_layout(params, pixels, nullptr, nullptr);
}

extern "C" size_t cpt_render_views_scratch_bytes(const cpt_view* views, uint32_t n_views,
                                                 const cpt_render_params* params)
{
    if (!views || n_views == 0 || n_views > CPT_MAX_VIEWS) return 0;
    uint64_t pixels = 0;
    for (uint32_t i = 0; i < n_views; ++i) pixels += (uint64_t)views[i].width * views[i].height;
    if (!params_ok(params, pixels)) return 0;
    return render_layout(params, pixels, nullptr, nullptr);
}

size_t cpt::render_hook_layout(const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void*,
                               uint32_t* capacity)
{
    if (!views || n_views == 0 || n_views > CPT_MAX_VIEWS || !params) return 0;
    uint64_t pixels = 0;
    for (uint32_t i = 0; i < n_views; ++i) pixels += (uint64_t)views[i].width * views[i].height;
    if (!params_ok(params, pixels)) return 0;
    const uint64_t cap = pixels * wave_samples(params, pixels);
    if (capacity) *capacity = std::max<uint32_t>(*capacity, (uint32_t)cap);
    return align_up((size_t)cap * 5 * sizeof(float4), 256);
}

extern "C" int cpt_render_views(const cpt_view* views, uint32_t n_views, const cpt_render_params* params,
                                void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                                cudaStream_t stream)
{
    CPT_RANGE("cpt_render_views");
    return cpt::cpt_render_views_hooked(views, n_views, params, scratch, scratch_bytes, ray_counts, status, nullptr,
                                        stream);
}

int cpt::cpt_render_views_hooked(const cpt_view* views, uint32_t n_views, const cpt_render_params* params,
                                 void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                                 const RenderHook* hook, cudaStream_t stream)
{
    if (!views || n_views == 0 || n_views > CPT_MAX_VIEWS || !params || !status) return CPT_ERR_INVALID_ARGUMENT;
    static Views vs;  // 14 KB: built on the host, passed by value to the kernels
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    if (!make_views(views, n_views, params->ref_grid, params->nee != 0, vs)) return CPT_ERR_INVALID_ARGUMENT;
    bool lights = false;
    for (uint32_t i = 0; i < n_views; ++i) lights |= views[i].scene->light_count > 0;
    return render_views(vs, lights, views[0].bvh->node_boxes, params, scratch, scratch_bytes, ray_counts, status, hook,
                        stream);
}

extern "C" int cpt_render(const cpt_bvh* bvh, const cpt_scene* scene, const cpt_camera* camera,
                          const cpt_render_params* params, void* accum, void* scratch, size_t scratch_bytes,
                          unsigned long long* ray_counts, uint32_t* status, cudaStream_t stream)
{
    CPT_RANGE("cpt_render");
    if (!bvh || !scene || !camera || !accum || !params || params->width == 0 || params->height == 0)
        return CPT_ERR_INVALID_ARGUMENT;
    const uint32_t ncam = camera_count(params);
    if (ncam > CPT_MAX_VIEWS) return CPT_ERR_INVALID_ARGUMENT;
    const size_t stride = cpt_accum_bytes(params->width, params->height, params->accum_mode);
    cpt_view views[CPT_MAX_VIEWS];
    for (uint32_t c = 0; c < ncam; ++c) {
        views[c].bvh = bvh;
        views[c].scene = scene;
        views[c].camera = camera[c];
        views[c].width = params->width;
        views[c].height = params->height;
        views[c].accum = static_cast<char*>(accum) + stride * c;
    }
    return cpt_render_views(views, ncam, params, scratch, scratch_bytes, ray_counts, status ? status : bvh->status,
                            stream);
}

extern "C" int cpt_resolve(const void* accum, uint32_t width, uint32_t height, uint32_t accum_mode, float* rgba,
                           cudaStream_t stream)
{
    CPT_RANGE("cpt_resolve");
    if (!accum || !rgba || width == 0 || height == 0 || accum_mode > CPT_ACCUM_F64) return CPT_ERR_INVALID_ARGUMENT;
    const uint32_t px = width * height;
    {
        CPT_PROF(K_RESOLVE, stream);
        k_resolve<<<(px + 255) / 256, 256, 0, stream>>>(accum, px, accum_mode, reinterpret_cast<float4*>(rgba));
    }
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}
