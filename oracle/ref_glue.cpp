// Host build of the reference's own LBVH builder and closest-hit traversal, used
// by the tests to pin the oracle restatement (oracle/cpt_oracle.c) and by
// bench.py as the timed CPU baseline. TEST INFRASTRUCTURE ONLY: nothing in the
// product links or calls this.
//
// The reference sources are compiled in place from the reference tree by
// oracle/Makefile (target `ref`), with oracle/ref_shim/host_compat.h force-included
// and thrust's OpenMP device system. Only the glue below is ours:
//  * ref_build   — calls the reference's CUDA::BVHBuilder::build
//                  (BVHBuilder.cu:207-269) unchanged. The key width is the
//                  reference's compile-time MortonIntType (BVHBuilder.h:7-8), which
//                  also sets the quantization grid (BVHBuilder.cu:10): libref.so is
//                  the shipped 30-bit configuration, libref64.so the 63-bit one.
//  * ref_trace   — CUDA::trace (trace.h:73-169) per ray, OpenMP over rays.
//  * ref_render  — the per-pixel integrator of cuda_path_tracer.cu:163-333,385-421
//                  restated over the reference's own CUDA::trace, CUDA::computeL
//                  (LightAlgorithms.h:12-20), CUDA::toHemisphere (math_util.h:56-67)
//                  and TriangleInfo::computeColor/computeNormal (TriangleInfo.h:39-50),
//                  with curand replaced by the shared Philox4x32-10 stream
//                  (oracle/cpt_rng.h); blinnPhongBRDF (cuda_path_tracer.cu:36-50)
//                  lives in a .cu that needs curand and is restated here.
// The 30-bit library compiles the builder where it lies; the 63-bit one compiles
// the same file staged next to BVHBuilder.h with its key alias switched to
// uint64_t (BVHBuilder.h:7-8), see oracle/Makefile.
#ifndef CPT_REF_BVHBUILDER
#define CPT_REF_BVHBUILDER "application/cuda/BVHBuilder.cu"
#endif
#include CPT_REF_BVHBUILDER
#include "application/cuda/LightAlgorithms.h"
#include "application/cuda/TriangleInfo.h"
#include "application/cuda/math_util.h"
#include <glm/gtx/compatibility.hpp>
#include "cpt_rng.h"

#include <cstdio>
#include <vector>
#include <unistd.h>
#include <omp.h>

// The reference defines these __constant__ descriptors in Scene.cu:8-11; trace.h
// reads g_geometryData, computeL reads nothing else.
GeometryData g_geometryData;
ShadingData g_shadingData;
LightingData g_lightingData;
MiscData g_miscData;

namespace {

// BVHBuilder::build prints the two root volumes on stdout (BVHBuilder.cu:263-264);
// callers of this library own stdout (bench.py prints one JSON line), so the
// builder's chatter is moved to stderr for the duration of a call.
struct StdoutToStderr {
    int saved;
    StdoutToStderr() { fflush(stdout); saved = dup(1); dup2(2, 1); }
    ~StdoutToStderr() { fflush(stdout); dup2(saved, 1); close(saved); }
};

BBox box_from(const float* b) { return BBox(glm::vec3(b[0], b[1], b[2]), glm::vec3(b[3], b[4], b[5])); }

}  // namespace

extern "C" {

int ref_sizeof_triangle(void) { return (int)sizeof(CUDA::Triangle); }
int ref_sizeof_bbox(void) { return (int)sizeof(BBox); }
int ref_sizeof_node(void) { return (int)sizeof(Node); }
int ref_sizeof_triangle_info(void) { return (int)sizeof(CUDA::TriangleInfo); }

// Builds the LBVH over n triangles (40-byte CUDA::Triangle records) with the
// host-provided enclosing box (min xyz, max xyz) and writes the reference-format
// outputs: Morton-sorted triangles, sorted keys, children, both parent arrays and
// the internal-node boxes. Returns 0, -1 for n < 2, -2 when bits is not this
// library's configured key width.
int ref_key_bits(void) { return sizeof(MortonIntType) == 8 ? 63 : 30; }

int ref_build(const void* tris_in, uint32_t n, const float* box, int bits,
              void* tris_out, void* keys_out, uint32_t* children, uint32_t* parents_leaf,
              uint32_t* parents_internal, float* node_boxes)
{
    if (n < 2) return -1;
    if (bits != ref_key_bits()) return -2;
    StdoutToStderr quiet;
    const CUDA::Triangle* in = static_cast<const CUDA::Triangle*>(tris_in);
    CUDA::DeviceSceneDescription desc;
    desc.triangles.assign(in, in + n);
    desc.enclosingBBox = box_from(box);
    CUDA::BVHBuilder builder;
    builder.build(desc, n);
    // Sorted keys: the encoder applied to the sorted triangles (same triangle, same key).
    morton_encoder<MortonIntType> enc(desc.enclosingBBox);
    MortonIntType* k = static_cast<MortonIntType*>(keys_out);
    for (uint32_t i = 0; i < n; ++i) k[i] = enc(desc.triangles[i]).value;
    thrust::copy(desc.triangles.begin(), desc.triangles.end(), static_cast<CUDA::Triangle*>(tris_out));
    thrust::copy(desc.children.begin(), desc.children.end(), reinterpret_cast<Node*>(children));
    thrust::copy(desc.parents[0].begin(), desc.parents[0].end(), parents_leaf);
    thrust::copy(desc.parents[1].begin(), desc.parents[1].end(), parents_internal);
    thrust::copy(desc.internalNodeBBoxes.begin(), desc.internalNodeBBoxes.end(), reinterpret_cast<BBox*>(node_boxes));
    return 0;
}

// Points the reference's g_geometryData at caller-owned reference-format arrays.
void ref_set_geometry(const void* sorted_tris, const uint32_t* children, const float* node_boxes, uint32_t n)
{
    g_geometryData = GeometryData(reinterpret_cast<const BBox*>(node_boxes),
                                  reinterpret_cast<const Node*>(children),
                                  static_cast<const CUDA::Triangle*>(sorted_tris), n);
}

// Closest hit for m rays (origin xyz, direction xyz) through CUDA::trace.
// Writes t (FLT_MAX on miss), the sorted-leaf triangle index (0xFFFFFFFF on miss)
// and the barycentric uv. threads <= 0 uses every OpenMP thread.
void ref_trace(const float* rays, uint32_t m, float* t_out, uint32_t* idx_out, float* uv_out, int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)m; ++i) {
        const float* r = rays + 6 * i;
        CUDA::Ray ray(glm::vec3(r[0], r[1], r[2]), glm::vec3(r[3], r[4], r[5]));
        TriangleIndex idx = INVALID_NODE_INDEX;
        glm::vec2 uv(0.0f);
        float t = CUDA::trace(ray, idx, uv);
        t_out[i] = t;
        idx_out[i] = idx;
        if (uv_out) { uv_out[2 * i] = uv.x; uv_out[2 * i + 1] = uv.y; }
    }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Integrator over the reference's device functions (compiled for the host).
// ---------------------------------------------------------------------------
namespace {

// cuda_path_tracer.cu:36-50
glm::vec3 blinn_phong_brdf(glm::vec3 Id, glm::vec3 kd, glm::vec3 Is, glm::vec3 ks,
                           glm::vec3 normal, glm::vec3 lightVec, glm::vec3 halfway, float shininess)
{
    float diffuseFactor = glm::max(glm::dot(normal, lightVec), 0.0f);
    glm::vec3 diffuse = Id * kd * diffuseFactor;
    float specFactor = std::pow(glm::max(glm::dot(normal, halfway), 0.0f), shininess);
    glm::vec3 specular(0.0f);
    if (shininess > 0.0 && diffuseFactor > 0.0f) specular = Is * ks * specFactor;
    return diffuse + specular;
}

struct RefShadeCtx {
    const CUDA::TriangleInfo* infos;
    const CUDA::DirectionalLight* lights;
    uint32_t lightCount;
    uint32_t bounces;
    float intensity;
    bool stratified;
};

const CUDA::TriangleInfo& info_of(const RefShadeCtx& c, TriangleIndex sortedIdx)
{
    return c.infos[g_geometryData.triangles[sortedIdx].infoIdx];
}

// cuda_path_tracer.cu:163-220 (primary vertex, untextured materials)
glm::vec3 primary_vertex(const RefShadeCtx& c, const CUDA::Ray& ray, TriangleIndex& idx,
                         glm::vec3& hitPos, glm::vec3& normal, glm::vec3& albedo, uint64_t* rays)
{
    glm::vec2 uv;
    float t = CUDA::trace(ray, idx, uv);
    ++rays[0];
    if (idx == INVALID_NODE_INDEX) return glm::vec3(0.0f);
    const CUDA::TriangleInfo& info = info_of(c, idx);
    hitPos = ray.direction * t + ray.origin;
    albedo = info.computeColor(uv);
    normal = info.computeNormal(uv);
    glm::vec3 emission = info.material.emission;
    if ((emission.r + emission.g + emission.b) > CUDA_EPSILON) {
        albedo = glm::vec3(1.0f);
        return emission;
    }
    glm::vec3 L(0.0f), color(0.0f);
    for (uint32_t i = 0; i < c.lightCount; ++i) {
        const CUDA::DirectionalLight& dl = c.lights[i];
        L += CUDA::computeL(hitPos, dl);
        ++rays[2];
        glm::vec3 view = -ray.direction;
        glm::vec3 halfway = 0.5f * (view - dl.direction);
        color += blinn_phong_brdf(L, albedo, L, glm::vec3(0.5f), normal, -dl.direction, halfway,
                                  info.material.specularity);
    }
    return color;
}

// cuda_path_tracer.cu:245-333
glm::vec3 path_trace(const RefShadeCtx& c, const CUDA::Ray& primary, uint32_t pixel, uint32_t frame,
                     uint32_t key0, uint32_t key1, uint64_t* rays)
{
    TriangleIndex idx;
    glm::vec3 hitPos, normal, albedo;
    glm::vec2 uv;
    CUDA::Ray cur = primary;
    glm::vec3 acc = primary_vertex(c, cur, idx, hitPos, normal, albedo, rays);
    glm::vec3 absorbed = albedo;
    if (idx == INVALID_NODE_INDEX) return glm::vec3(0.0f);
    for (uint32_t i = 0; i < c.bounces; ++i) {
        cur.origin = hitPos + normal * CUDA_EPSILON5;
        float u0, u1;
        cpt_rng_bounce_uniforms(key0, key1, pixel, frame, i, 0u, &u0, &u1);
        glm::vec2 rnd(u0, u1);
        if (c.stratified && i == 0) {
            const int extent = 8;
            uint32_t pos1D = frame % (extent * extent);
            rnd = glm::vec2((int(pos1D % extent) + u0) / extent, (int(pos1D / extent) + u1) / extent);
        }
        float s, co;
        cpt_sincos_turns(rnd.y, &s, &co);
        float r = sqrtf(rnd.x);
        cur.direction = glm::vec3(r * co, r * s, sqrtf(1.0f - rnd.x));
        cur.direction = CUDA::toHemisphere(cur.direction, normal);
        float t = CUDA::trace(cur, idx, uv);
        ++rays[1];
        if (idx == INVALID_NODE_INDEX) break;
        hitPos = cur.direction * t + cur.origin;
        const CUDA::TriangleInfo& info = info_of(c, idx);
        albedo = info.computeColor(uv);
        normal = info.computeNormal(uv);
        glm::vec3 L(0.0f);
        glm::vec3 emission = info.material.emission;
        if ((emission.r + emission.g + emission.b) > CUDA_EPSILON) {
            L = emission * glm::max(glm::dot(-cur.direction, normal), 0.0f);
            albedo = glm::vec3(1.0f);
        } else {
            for (uint32_t l = 0; l < c.lightCount; ++l) {
                const CUDA::DirectionalLight& dl = c.lights[l];
                L += CUDA::computeL(hitPos, dl) * glm::max(glm::dot(-dl.direction, normal), 0.0f);
                ++rays[2];
            }
        }
        absorbed *= albedo;
        acc += absorbed * L * c.intensity;
    }
    return acc;
}

}  // namespace

extern "C" {

// Renders `spp` samples (global sample indices frame0 .. frame0+spp-1) of a
// width x height image, rows [row0, row1), accumulating each pixel's samples in
// sample order into sum_out (3 floats per pixel of the row range, plain f32 sum).
// cam = eye xyz + four corner directions (00, 10, 11, 01) as in
// CUDAPathTracer::setPrimaryRays. ray_counts[3] receives primary / extension /
// shadow rays traced. Needs ref_set_geometry first.
int ref_render(const void* infos, const void* lights, uint32_t light_count,
               uint32_t width, uint32_t height, uint32_t row0, uint32_t row1,
               uint32_t spp, uint32_t frame0, uint32_t bounces, float intensity, int stratified,
               uint32_t key0, uint32_t key1, const float* cam, float* sum_out,
               uint64_t* ray_counts, int threads)
{
    if (threads > 0) omp_set_num_threads(threads);
    RefShadeCtx c{static_cast<const CUDA::TriangleInfo*>(infos),
                  static_cast<const CUDA::DirectionalLight*>(lights), light_count, bounces, intensity,
                  stratified != 0};
    glm::vec3 eye(cam[0], cam[1], cam[2]);
    glm::vec3 d00(cam[3], cam[4], cam[5]), d10(cam[6], cam[7], cam[8]);
    glm::vec3 d11(cam[9], cam[10], cam[11]), d01(cam[12], cam[13], cam[14]);
    uint64_t tot[3] = {0, 0, 0};
#pragma omp parallel
    {
        uint64_t local[3] = {0, 0, 0};
#pragma omp for schedule(dynamic, 16)
        for (long p = (long)row0 * width; p < (long)row1 * width; ++p) {
            uint32_t x = (uint32_t)(p % width), y = (uint32_t)(p / width);
            glm::vec3 sum(0.0f);
            for (uint32_t s = 0; s < spp; ++s) {
                // cuda_path_tracer.cu:404-407 with lerpDirection :376-379
                glm::vec2 tc(x / (float)width, y / (float)height);
                CUDA::Ray ray;
                ray.direction = glm::lerp(glm::lerp(d00, d10, tc.x), glm::lerp(d01, d11, tc.x), tc.y);
                ray.origin = eye;
                sum += path_trace(c, ray, (uint32_t)p, frame0 + s, key0, key1, local);
            }
            float* o = sum_out + 3 * (p - (long)row0 * width);
            o[0] = sum.x; o[1] = sum.y; o[2] = sum.z;
        }
#pragma omp critical
        { tot[0] += local[0]; tot[1] += local[1]; tot[2] += local[2]; }
    }
    if (ray_counts) { ray_counts[0] = tot[0]; ray_counts[1] = tot[1]; ray_counts[2] = tot[2]; }
    return 0;
}

// The same integrator over an arbitrary list of rows (e.g. every k-th row of the
// frame, a sample spread over the whole image), each pixel's samples summed in
// sample order in float64 (the device's FP64 accumulator adds the same float
// radiance values in the same order). sum_out: 3 doubles per pixel, rows in list
// order. Returns -1 for a row outside the image. Needs ref_set_geometry first.
int ref_render_rows(const void* infos, const void* lights, uint32_t light_count,
                    uint32_t width, uint32_t height, const uint32_t* rows, uint32_t row_count,
                    uint32_t spp, uint32_t frame0, uint32_t bounces, float intensity, int stratified,
                    uint32_t key0, uint32_t key1, const float* cam, double* sum_out,
                    uint64_t* ray_counts, int threads)
{
    if (!rows || !sum_out) return -1;
    for (uint32_t r = 0; r < row_count; ++r)
        if (rows[r] >= height) return -1;
    if (threads > 0) omp_set_num_threads(threads);
    RefShadeCtx c{static_cast<const CUDA::TriangleInfo*>(infos),
                  static_cast<const CUDA::DirectionalLight*>(lights), light_count, bounces, intensity,
                  stratified != 0};
    glm::vec3 eye(cam[0], cam[1], cam[2]);
    glm::vec3 d00(cam[3], cam[4], cam[5]), d10(cam[6], cam[7], cam[8]);
    glm::vec3 d11(cam[9], cam[10], cam[11]), d01(cam[12], cam[13], cam[14]);
    uint64_t tot[3] = {0, 0, 0};
    const long total = (long)row_count * width;
#pragma omp parallel
    {
        uint64_t local[3] = {0, 0, 0};
#pragma omp for schedule(dynamic, 16)
        for (long q = 0; q < total; ++q) {
            uint32_t x = (uint32_t)(q % width), y = rows[q / width];
            long p = (long)y * width + x;
            double sum[3] = {0.0, 0.0, 0.0};
            for (uint32_t s = 0; s < spp; ++s) {
                // cuda_path_tracer.cu:404-407 with lerpDirection :376-379
                glm::vec2 tc(x / (float)width, y / (float)height);
                CUDA::Ray ray;
                ray.direction = glm::lerp(glm::lerp(d00, d10, tc.x), glm::lerp(d01, d11, tc.x), tc.y);
                ray.origin = eye;
                glm::vec3 v = path_trace(c, ray, (uint32_t)p, frame0 + s, key0, key1, local);
                sum[0] += (double)v.x; sum[1] += (double)v.y; sum[2] += (double)v.z;
            }
            double* o = sum_out + 3 * q;
            o[0] = sum[0]; o[1] = sum[1]; o[2] = sum[2];
        }
#pragma omp critical
        { tot[0] += local[0]; tot[1] += local[1]; tot[2] += local[2]; }
    }
    if (ray_counts) { ray_counts[0] = tot[0]; ray_counts[1] = tot[1]; ray_counts[2] = tot[2]; }
    return 0;
}

}  // extern "C"
