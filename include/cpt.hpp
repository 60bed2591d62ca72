/* C++ mirror of the reference's hot-path classes, header-only, over the C ABI of
 * cpt.h. A caller of the reference's CUDA::BVHBuilder / CUDAPathTracer
 * (source/application/cuda/BVHBuilder.h:12-19, cuda_path_tracer.h:13-40) keeps its
 * call sites: the same class and method names, the same argument meaning, scene
 * descriptions with the same members (DeviceSceneDescription.h:13-21,
 * HostSceneDescription.h:10-17) — with cpt::DeviceVector standing in for
 * thrust::device_vector and plain float triples for glm::vec3.
 *
 * Errors: the reference prints CUDA errors and carries on (cuda_common.h:4-12). By
 * default these classes do the same (message on stderr, status kept in
 * cpt::last_error()); cpt::error_policy() = cpt::OnError::Throw turns a failed call
 * into a std::runtime_error instead. */
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>
#include "cpt.h"

namespace cpt {

enum class OnError { Report, Throw };

inline OnError& error_policy()
{
    static OnError policy = OnError::Report;
    return policy;
}

inline int& last_error()
{
    static int code = CPT_OK;
    return code;
}

inline const char* status_text(int code)
{
    switch (code) {
    case CPT_OK: return "ok";
    case CPT_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CPT_ERR_CUDA: return "CUDA runtime error";
    case CPT_ERR_SCRATCH_TOO_SMALL: return "scratch buffer too small";
    case CPT_ERR_NONFINITE_INPUT: return "non-finite vertex coordinate";
    case CPT_ERR_DEVICE_TIMEOUT: return "device-side wait timed out";
    case CPT_ERR_STACK_OVERFLOW: return "traversal stack overflow";
    case CPT_ERR_CHECK_FAILED: return "root box volume differs from the enclosing box";
    case CPT_ERR_NO_DEVICE: return "no CUDA device";
    case CPT_ERR_BAD_INDEX: return "device-side index out of range";
    case CPT_ERR_TREE_TOO_DEEP: return "tree taller than the traversal stack";
    default: return "unknown status";
    }
}

// Returns true on CPT_OK; otherwise records the code and reports or throws.
inline bool check(int code, const char* what)
{
    if (code == CPT_OK) return true;
    last_error() = code;
    const std::string msg = std::string(what) + ": " + status_text(code) + " (" + std::to_string(code) + ")";
    if (error_policy() == OnError::Throw) throw std::runtime_error(msg);
    std::fprintf(stderr, "%s\n", msg.c_str());
    return false;
}

inline bool check_cuda(cudaError_t e, const char* what)
{
    return check(e == cudaSuccess ? CPT_OK : CPT_ERR_CUDA, what);
}

// The members thrust::device_vector gives the reference's callers: resize, size,
// data; plus host transfers.
template <typename T>
class DeviceVector {
public:
    DeviceVector() = default;
    explicit DeviceVector(size_t n) { resize(n); }
    ~DeviceVector() { release(); }
    DeviceVector(const DeviceVector&) = delete;
    DeviceVector& operator=(const DeviceVector&) = delete;
    DeviceVector(DeviceVector&& o) noexcept { swap(o); }
    DeviceVector& operator=(DeviceVector&& o) noexcept
    {
        swap(o);
        return *this;
    }

    void resize(size_t n)
    {
        if (n <= cap_) {
            size_ = n;
            return;
        }
        release();
        void* p = nullptr;
        if (!check_cuda(cudaMalloc(&p, n * sizeof(T)), "DeviceVector::resize")) return;
        ptr_ = static_cast<T*>(p);
        cap_ = size_ = n;
    }
    T* data() { return ptr_; }
    const T* data() const { return ptr_; }
    size_t size() const { return size_; }
    bool empty() const { return size_ == 0; }

    void assign(const T* host, size_t n, cudaStream_t stream = 0)
    {
        resize(n);
        if (n && ptr_) {
            check_cuda(cudaMemcpyAsync(ptr_, host, n * sizeof(T), cudaMemcpyHostToDevice, stream), "DeviceVector::assign");
            check_cuda(cudaStreamSynchronize(stream), "DeviceVector::assign");
        }
    }
    std::vector<T> to_host(cudaStream_t stream = 0) const
    {
        std::vector<T> out(size_);
        if (size_ && ptr_) {
            check_cuda(cudaMemcpyAsync(out.data(), ptr_, size_ * sizeof(T), cudaMemcpyDeviceToHost, stream),
                       "DeviceVector::to_host");
            check_cuda(cudaStreamSynchronize(stream), "DeviceVector::to_host");
        }
        return out;
    }

private:
    void release()
    {
        if (ptr_) cudaFree(ptr_);
        ptr_ = nullptr;
        size_ = cap_ = 0;
    }
    void swap(DeviceVector& o)
    {
        std::swap(ptr_, o.ptr_);
        std::swap(size_, o.size_);
        std::swap(cap_, o.cap_);
    }
    T* ptr_ = nullptr;
    size_t size_ = 0, cap_ = 0;
};

constexpr int LEAF_PARENTS_IDX = 0;      // DeviceSceneDescription.h:8
constexpr int INTERNAL_PARENTS_IDX = 1;  // DeviceSceneDescription.h:9

struct Vec3 {
    float x, y, z;
};

// CUDA::Ray (geometry.h:11-18)
struct Ray {
    Vec3 origin;
    Vec3 direction;
};

// CUDA::DeviceSceneDescription (DeviceSceneDescription.h:13-21)
struct DeviceSceneDescription {
    DeviceVector<uint32_t> children;  // Node words
    DeviceVector<uint32_t> parents[2];
    DeviceVector<cpt_triangle> triangles;
    DeviceVector<cpt_bbox> internalNodeBBoxes;
    DeviceVector<cpt_triangle_info> triangleInfo;
    cpt_bbox enclosingBBox{};
};

// CUDA::HostSceneDescription (HostSceneDescription.h:10-17)
struct HostSceneDescription {
    std::vector<cpt_triangle> triangles;
    std::vector<cpt_triangle_info> triangleInfo;
    cpt_bbox enclosingBBox{};
    std::vector<cpt_dir_light> dirLights;
};

// CUDA::BVHBuilder (BVHBuilder.h:12-19, BVHBuilder.cu:207-269). build() permutes
// outSceneDesc.triangles into Morton order in place and fills children, parents and
// internalNodeBBoxes; kMortonBits is the reference's MortonIntType (uint32_t -> 30,
// uint64_t -> 63). The builder keeps its scratch (as the reference keeps
// m_mortonCodes) and the traversal records, which bvh() exposes for cpt_trace.
template <int kMortonBits = 30>
class BVHBuilder {
    static_assert(kMortonBits == 30 || kMortonBits == 63, "30- or 63-bit Morton keys");

public:
    void build(DeviceSceneDescription& outSceneDesc, size_t triangleCount, cudaStream_t stream = 0)
    {
        const uint32_t n = static_cast<uint32_t>(triangleCount);
        if (n < 2 || outSceneDesc.triangles.size() < n) {
            check(CPT_ERR_INVALID_ARGUMENT, "BVHBuilder::build");
            return;
        }
        outSceneDesc.children.resize(n - 1);
        outSceneDesc.parents[LEAF_PARENTS_IDX].resize(n);
        outSceneDesc.parents[INTERNAL_PARENTS_IDX].resize(n - 1);
        outSceneDesc.internalNodeBBoxes.resize(n - 1);
        m_keys.resize(size_t(n) * (kMortonBits == 30 ? 4 : 8));
        m_nodes.resize(size_t(n - 1) * 96);
        m_status.resize(4);
        m_scratch.resize(cpt_lbvh_scratch_bytes(n, kMortonBits));
        cpt_bvh bvh{};
        bvh.n = n;
        bvh.morton_bits = kMortonBits;
        bvh.tris = outSceneDesc.triangles.data();
        bvh.keys = m_keys.data();
        bvh.children = outSceneDesc.children.data();
        bvh.parents_leaf = outSceneDesc.parents[LEAF_PARENTS_IDX].data();
        bvh.parents_internal = outSceneDesc.parents[INTERNAL_PARENTS_IDX].data();
        bvh.node_boxes = outSceneDesc.internalNodeBBoxes.data();
        bvh.nodes = m_nodes.data();
        bvh.status = m_status.data();
        const cpt_bbox& b = outSceneDesc.enclosingBBox;
        const float box[6] = {b.min[0], b.min[1], b.min[2], b.max[0], b.max[1], b.max[2]};
        // tris_in == bvh.tris: sorted in place; CPT_BUILD_CHECK is the root-volume
        // check the reference asserts (BVHBuilder.cu:258-265)
        if (check(cpt_lbvh_build(bvh.tris, n, box, kMortonBits, &bvh, m_scratch.data(), m_scratch.size(),
                                 CPT_BUILD_CHECK, stream),
                  "BVHBuilder::build"))
            m_bvh = bvh;
    }

    const cpt_bvh& bvh() const { return m_bvh; }

private:
    DeviceVector<uint8_t> m_keys, m_nodes, m_scratch;
    DeviceVector<uint32_t> m_status;
    cpt_bvh m_bvh{};
};

// CUDAPathTracer (cuda_path_tracer.h:13-40) over cpt_tracer_*. The GL surface of
// setScreenTexture is replaced by readImage (a headless RGBA32F copy).
class CUDAPathTracer {
public:
    explicit CUDAPathTracer(int mortonBits = 30) { check(cpt_tracer_create(&m_t, mortonBits), "CUDAPathTracer"); }
    ~CUDAPathTracer() { cpt_tracer_destroy(m_t); }
    CUDAPathTracer(const CUDAPathTracer&) = delete;
    CUDAPathTracer& operator=(const CUDAPathTracer&) = delete;

    void setPrimaryRays(const Ray& ray00, const Ray& ray10, const Ray& ray11, const Ray& ray01)
    {
        // only the directions are used, as in cuda_path_tracer.cu:366-374
        const float d[12] = {ray00.direction.x, ray00.direction.y, ray00.direction.z,
                             ray10.direction.x, ray10.direction.y, ray10.direction.z,
                             ray11.direction.x, ray11.direction.y, ray11.direction.z,
                             ray01.direction.x, ray01.direction.y, ray01.direction.z};
        check(cpt_tracer_set_primary_rays(m_t, d), "CUDAPathTracer::setPrimaryRays");
    }
    void setEyePos(const Vec3& eyePos)
    {
        const float e[3] = {eyePos.x, eyePos.y, eyePos.z};
        check(cpt_tracer_set_eye(m_t, e), "CUDAPathTracer::setEyePos");
    }
    void raytrace(int screenWidth, int screenHeight)
    {
        if (screenWidth <= 0 || screenHeight <= 0) {
            check(CPT_ERR_INVALID_ARGUMENT, "CUDAPathTracer::raytrace");
            return;
        }
        if (!check(cpt_tracer_raytrace(m_t, uint32_t(screenWidth), uint32_t(screenHeight), 1), "CUDAPathTracer::raytrace"))
            return;
        if (!m_screen) return;
        // the reference's raytrace_kernel writes every pixel's running value into the screen
        // surface (cuda_path_tracer.cu:416-420); here the resolved image goes into the array
        const size_t row = size_t(screenWidth) * 4 * sizeof(float);
        m_image.resize(size_t(screenWidth) * size_t(screenHeight) * 4);
        if (!m_image.data() || !check(cpt_tracer_resolve(m_t, m_image.data()), "CUDAPathTracer::raytrace")) return;
        check_cuda(cudaMemcpy2DToArrayAsync(m_screen, 0, 0, m_image.data(), row, row, size_t(screenHeight),
                                            cudaMemcpyDeviceToDevice, cpt_tracer_stream(m_t)),
                   "CUDAPathTracer::raytrace");
    }
    // CUDAPathTracer::setScreenTexture (cuda_path_tracer.h:18): a float4 (RGBA32F) array of
    // the screen size, e.g. a mapped OpenGL texture, that every raytrace() updates with the
    // accumulated image on the tracer's stream. nullptr: no screen array.
    void setScreenTexture(const cudaArray_t* screenArray) { m_screen = screenArray ? *screenArray : nullptr; }
    void upload(const HostSceneDescription& sceneDesc)
    {
        const cpt_bbox& b = sceneDesc.enclosingBBox;
        const float box[6] = {b.min[0], b.min[1], b.min[2], b.max[0], b.max[1], b.max[2]};
        check(cpt_tracer_upload(m_t, sceneDesc.triangles.data(), uint32_t(sceneDesc.triangles.size()),
                                sceneDesc.triangleInfo.data(), uint32_t(sceneDesc.triangleInfo.size()),
                                sceneDesc.dirLights.empty() ? nullptr : sceneDesc.dirLights.data(),
                                uint32_t(sceneDesc.dirLights.size()), box),
              "CUDAPathTracer::upload");
    }
    void resetFrames() { cpt_tracer_reset_frames(m_t); }

    // PathTracerSettings::GI (PathTracingSettings.h:26-28) and the random seed
    void setSettings(uint32_t indirectBounceCount, float indirectIntensity, bool useStratifiedSampling,
                     uint64_t seed = 0, uint32_t accumMode = CPT_ACCUM_KAHAN)
    {
        check(cpt_tracer_set_settings(m_t, indirectBounceCount, indirectIntensity, useStratifiedSampling ? 1u : 0u,
                                      uint32_t(seed), uint32_t(seed >> 32), accumMode),
              "CUDAPathTracer::setSettings");
    }
    // extensions without a reference counterpart: next-event estimation, split and wide traversal trees
    void setNextEventEstimation(bool on) { check(cpt_tracer_set_nee(m_t, on ? 1u : 0u), "CUDAPathTracer::setNextEventEstimation"); }
    void setSplit(float extraRatio, uint32_t flags = 0)
    {
        check(cpt_tracer_set_split(m_t, extraRatio, flags), "CUDAPathTracer::setSplit");
    }
    // sah: the surface-area collapse (a longer build, a faster render; a scene uploaded once)
    void setWide(bool on, bool sah = false)
    {
        check(cpt_tracer_set_wide(m_t, on ? (sah ? 2u : 1u) : 0u), "CUDAPathTracer::setWide");
    }
    // the accumulated image, width x height RGBA32F (replaces the GL surface)
    std::vector<float> readImage(int screenWidth, int screenHeight)
    {
        std::vector<float> img(size_t(screenWidth) * size_t(screenHeight) * 4);
        check(cpt_tracer_read_image(m_t, img.data()), "CUDAPathTracer::readImage");
        return img;
    }
    uint32_t frame() const { return cpt_tracer_frame(m_t); }
    cpt_tracer* handle() { return m_t; }

private:
    cpt_tracer* m_t = nullptr;
    cudaArray_t m_screen = nullptr;
    DeviceVector<float> m_image;  // the resolved image on its way into m_screen
};

}  // namespace cpt
