// BVH heat map (cpt_bvh_heatmap): the reference's debug visualisation
// CUDA::computeBVHColor (source/application/cuda/visualization.h:19-66), which
// the reference app never calls. Per pixel, the primary ray of the camera is
// pushed through every internal node whose box it hits (no pruning, no triangle
// tests); each such node adds base_color once. The stack is the reference's
// 64 entries; as there, the walk stops when it is full.
#include <cuda_runtime.h>
#include "cpt.h"
#include "cpt_internal.h"
#include "traverse.cuh"

namespace cpt {

struct HeatCam {
    float eye[3];
    float dirs[4][3];
};

__global__ void __launch_bounds__(128) k_heatmap(const float4* __restrict__ nodes, HeatCam cam, uint32_t width,
                                                 uint32_t height, float bx, float by, float bz,
                                                 float4* __restrict__ rgba, uint32_t* __restrict__ counts)
{
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    if (px >= width * height) return;
    const uint32_t x = px % width, y = px / width;
    const float tx = __fdiv_rn(__uint2float_rn(x), __uint2float_rn(width));
    const float ty = __fdiv_rn(__uint2float_rn(y), __uint2float_rn(height));
    const f3 c00 = ld3(cam.dirs[0]), c10 = ld3(cam.dirs[1]), c11 = ld3(cam.dirs[2]), c01 = ld3(cam.dirs[3]);
    const f3 d = mix3(mix3(c00, c10, tx), mix3(c01, c11, tx), ty);
    const f3 o = ld3(cam.eye);
    const f3 dinv = mk3(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
    const bool finite = isfinite(dinv.x) && isfinite(dinv.y) && isfinite(dinv.z);
    uint32_t stack[CPT_TRAVERSAL_STACK];
    int sp = 0;
    stack[sp++] = 0;  // the root
    float ax = 0.f, ay = 0.f, az = 0.f;
    uint32_t count = 0;
    bool full = false;
    while (sp > 0 && !full) {
        const uint32_t cur = stack[--sp];
        const float* w = reinterpret_cast<const float*>(nodes + kNodeFloat4 * (size_t)cur);
        const uint32_t word = __float_as_uint(__ldg(w + 20));
        for (int side = 0; side < 2 && !full; ++side) {
            if (!((word >> side) & 1u)) continue;  // only internal children have boxes
            const float* s = w + 10 * side;
            if (slab_test(o, dinv, finite, __ldg(s), __ldg(s + 1), __ldg(s + 2), __ldg(s + 3), __ldg(s + 4),
                          __ldg(s + 5)) < FLT_MAX) {
                stack[sp++] = (word >> 2) + (uint32_t)side;
                ax = __fadd_rn(ax, bx);
                ay = __fadd_rn(ay, by);
                az = __fadd_rn(az, bz);
                ++count;
            }
            full = sp == CPT_TRAVERSAL_STACK;
        }
    }
    rgba[px] = make_float4(ax, ay, az, 1.0f);
    if (counts) counts[px] = count;
}

}  // namespace cpt

using namespace cpt;

extern "C" int cpt_bvh_heatmap(const cpt_bvh* bvh, const cpt_camera* camera, uint32_t width, uint32_t height,
                               const float base_color[3], float* rgba, uint32_t* node_counts, cudaStream_t stream)
{
    CPT_RANGE("cpt_bvh_heatmap");
    if (!bvh || !bvh->nodes || !camera || !base_color || !rgba || width == 0 || height == 0) return CPT_ERR_INVALID_ARGUMENT;
    if ((uint64_t)width * height >= (1ull << 31) || (reinterpret_cast<uintptr_t>(rgba) & 15)) return CPT_ERR_INVALID_ARGUMENT;
    HeatCam hc;
    for (int a = 0; a < 3; ++a) hc.eye[a] = camera->eye[a];
    for (int c = 0; c < 4; ++c)
        for (int a = 0; a < 3; ++a) hc.dirs[c][a] = camera->dirs[c][a];
    const uint32_t px = width * height;
    k_heatmap<<<(px + 127) / 128, 128, 0, stream>>>(static_cast<const float4*>(bvh->nodes), hc, width, height,
                                                     base_color[0], base_color[1], base_color[2],
                                                     reinterpret_cast<float4*>(rgba), node_counts);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}

// ---------------------------------------------------------------------------
// Per-frame deformation of a synthetic mesh (the deforming-mesh benchmark): every
// vertex moves along its direction from the origin, v_a += amp * sin(omega * v_a +
// phase) * n_a, n = v / |v|. Shared vertices of the soup move identically.
// ---------------------------------------------------------------------------
namespace cpt {
__global__ void __launch_bounds__(256) k_deform(const float* __restrict__ rest, float* __restrict__ out, uint32_t n,
                                                float amp, float omega, float phase)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* s = rest + 10ull * i;
    float* d = out + 10ull * i;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const float x = s[3 * v], y = s[3 * v + 1], z = s[3 * v + 2];
        const float inv = rsqrtf(fmaxf(x * x + y * y + z * z, 1e-30f));
        d[3 * v] = x + amp * __sinf(omega * x + phase) * x * inv;
        d[3 * v + 1] = y + amp * __sinf(omega * y + phase) * y * inv;
        d[3 * v + 2] = z + amp * __sinf(omega * z + phase) * z * inv;
    }
    d[9] = s[9];
}
}  // namespace cpt

extern "C" int cpt_scene_deform(const cpt_triangle* rest, cpt_triangle* out, uint32_t n, float amplitude, float omega,
                                float phase, cudaStream_t stream)
{
    CPT_RANGE("cpt_scene_deform");
    if (!rest || !out || n == 0) return CPT_ERR_INVALID_ARGUMENT;
    k_deform<<<(n + 255) / 256, 256, 0, stream>>>(reinterpret_cast<const float*>(rest), reinterpret_cast<float*>(out), n,
                                                   amplitude, omega, phase);
    CPT_LAUNCH_CHECK();
    return CPT_OK;
}
