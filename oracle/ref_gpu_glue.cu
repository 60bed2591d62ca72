// The reference's own GPU LBVH build, compiled from its sources for sm_100a, so that
// it can be timed on the same B200 beside this library's build and its outputs
// compared with the library's. TEST AND BASELINE INFRASTRUCTURE ONLY: used by the
// tests and by the benchmark's baseline leg; nothing in the product links it.
//
// What runs is CUDA::BVHBuilder::build (source/application/cuda/BVHBuilder.cu:207-269)
// as shipped: 30-bit Morton keys (BVHBuilder.h:8), thrust::transform for the codes,
// thrust::sort_by_key permuting the 40-B triangles in place, the radix-tree kernel
// (:107-201) and the atomic refit (:39-98) through thrust algorithms, together with
// its per-build resizes, temporary allocations, the 2-pointer cudaMalloc/cudaMemcpy
// (:238-242) and the root-box read-back (:258-265). Only the QueryManager timer is a
// no-op stand-in (oracle/ref_shim). BBox.cpp's host/device methods are compiled in
// the same translation unit, as the reference's build compiles them for the device.
// The reference declares CUDA::swap(T&, T&) as a __device__-only template
// (application/cuda/util.h:14-20). This toolkit's thrust swaps a vector's storage with an
// unqualified swap, so for vectors of CUDA:: types (CUDA::Triangle, CUDA::TriangleInfo)
// argument-dependent lookup selects that device-only function in host code, whose host
// copy ends the process (the reference's own Scene::upload assignment takes this path).
// These overloads for thrust's vector iterators and allocators are more specialized, so
// overload resolution prefers them, and they run on the host.
#include <thrust/device_vector.h>
namespace CUDA
{
template <typename Ptr>
__host__ __device__ inline void swap(thrust::detail::normal_iterator<Ptr>& a, thrust::detail::normal_iterator<Ptr>& b)
{
    thrust::detail::normal_iterator<Ptr> t = a;
    a = b;
    b = t;
}
template <typename T>
__host__ __device__ inline void swap(thrust::device_allocator<T>& a, thrust::device_allocator<T>& b)
{
    thrust::device_allocator<T> t = a;
    a = b;
    b = t;
}
}  // namespace CUDA

#include "engine/geometry/BBox.cpp"
#include "application/cuda/BVHBuilder.cu"
// The reference's path tracer (raytrace_kernel and the shading it calls,
// cuda_path_tracer.cu:36-421) with the constant-memory scene descriptors it reads
// (declared extern in Globals.h). As in the reference's build, the library is compiled
// with relocatable device code and the descriptors are defined once, here, as
// Scene.cu:8-11 defines them. Its host-side helpers come along: the mt19937 frame seeds
// (Random.cpp) and, as stand-ins without SDL / ImGui, the timer and GUI settings types
// (oracle/ref_shim/engine/util/Timer.h, engine/gui/GUISettings.h).
#include "engine/util/Random.cpp"
#include "application/cuda/cuda_path_tracer.cu"

__constant__ GeometryData g_geometryData;
__constant__ ShadingData g_shadingData;
__constant__ LightingData g_lightingData;
__constant__ MiscData g_miscData;

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <execinfo.h>
#include <unistd.h>

namespace {

// BVHBuilder::build prints the two root volumes on stdout (BVHBuilder.cu:263-264);
// the benchmark owns stdout (one JSON line), so the builder's lines go to stderr.
struct StdoutToStderr {
    int saved;
    StdoutToStderr() { std::cout.flush(); fflush(stdout); saved = dup(1); dup2(2, 1); }
    ~StdoutToStderr() { std::cout.flush(); fflush(stdout); dup2(saved, 1); close(saved); }
};

// With CPT_REFGPU_TRACE set, each step of a call is reported on stderr, and a process
// exit that passes through exit() prints where it came from (diagnostics of the child
// process that runs this library).
bool trace_on()
{
    static const bool on = getenv("CPT_REFGPU_TRACE") != nullptr;
    return on;
}

void trace(const char* what)
{
    if (!trace_on()) return;
    fprintf(stderr, "refgpu: %s\n", what);
    fflush(stderr);
}

void exit_backtrace()
{
    void* frames[32];
    const int k = backtrace(frames, 32);
    fprintf(stderr, "refgpu: process exit via exit(); backtrace:\n");
    backtrace_symbols_fd(frames, k, 2);
}

// trace() with the device's last error
void trace_error(const char* what)
{
    if (!trace_on()) return;
    const cudaError_t e = cudaGetLastError();
    fprintf(stderr, "refgpu: %s (%s)\n", what, cudaGetErrorString(e));
    fflush(stderr);
}

template <typename V>
void release(V& v)
{
    v.clear();
    v.shrink_to_fit();
}

// A failed CUDA call: reported, and the runtime's last error cleared so that the
// thrust vectors' destructors on the way out do not see it and throw.
int fail(cudaError_t e, const char* what)
{
    fprintf(stderr, "refgpu: %s: %s\n", what, cudaGetErrorName(e));
    cudaGetLastError();
    return -2;
}

struct ExitTrace {
    ExitTrace()
    {
        if (trace_on()) atexit(exit_backtrace);
    }
} g_exit_trace;

}  // namespace

extern "C" {

#define REFGPU_API __attribute__((visibility("default")))

REFGPU_API int refgpu_key_bits(void) { return sizeof(MortonIntType) == 8 ? 63 : 30; }

// Uploads n triangles (host, 40-B CUDA::Triangle records) and the enclosing box
// (host, min xyz, max xyz), runs one untimed warm-up build, then `reps` builds, each
// from the unsorted triangles (restoring the input order is outside the timed span).
// Per build, CUDA events on the legacy default stream (the one the builder uses)
// bracket BVHBuilder::build; the host wall time of the call is taken beside them.
// Outputs: mean and least event time (ms), mean wall time (ms); when the array
// pointers are non-null, the last build's sorted triangles, Node words, both parent
// arrays and the internal-node boxes (24 B each) are copied to host memory.
// Returns 0, -1 for bad arguments, -2 for a CUDA error, -3 when thrust threw.
static int refgpu_build_impl(const void* tris_host, uint32_t n, const float* box, int reps, float* ms_mean,
                             float* ms_min, float* wall_ms_mean, void* tris_out, uint32_t* children_out,
                             uint32_t* parents_leaf_out, uint32_t* parents_internal_out, float* boxes_out);

// thrust reports CUDA failures by throwing; nothing may unwind through this C interface,
// so an exception becomes -3 with its message on stderr
REFGPU_API int refgpu_build(const void* tris_host, uint32_t n, const float* box, int reps, float* ms_mean,
                            float* ms_min, float* wall_ms_mean, void* tris_out, uint32_t* children_out,
                            uint32_t* parents_leaf_out, uint32_t* parents_internal_out, float* boxes_out)
{
    try {
        return refgpu_build_impl(tris_host, n, box, reps, ms_mean, ms_min, wall_ms_mean, tris_out, children_out,
                                 parents_leaf_out, parents_internal_out, boxes_out);
    } catch (const std::exception& e) {
        fprintf(stderr, "refgpu_build: %s\n", e.what());
    } catch (...) {
        fprintf(stderr, "refgpu_build: unknown exception\n");
    }
    return -3;
}

}  // extern "C"

static int refgpu_build_impl(const void* tris_host, uint32_t n, const float* box, int reps, float* ms_mean,
                             float* ms_min, float* wall_ms_mean, void* tris_out, uint32_t* children_out,
                             uint32_t* parents_leaf_out, uint32_t* parents_internal_out, float* boxes_out)
{
    if (!tris_host || !box || n < 2 || reps < 1) return -1;
    trace("build: start");
    StdoutToStderr quiet;
    const CUDA::Triangle* in = static_cast<const CUDA::Triangle*>(tris_host);
    thrust::device_vector<CUDA::Triangle> source(in, in + n);
    trace("build: triangles uploaded");
    CUDA::DeviceSceneDescription desc;
    desc.triangles = source;
    desc.enclosingBBox = BBox(glm::vec3(box[0], box[1], box[2]), glm::vec3(box[3], box[4], box[5]));
    CUDA::BVHBuilder builder;
    builder.build(desc, n);  // warm-up: first allocations, thrust's temporary storage
    trace("build: warm-up build done");
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -2;
    double sum = 0.0, wall = 0.0;
    float least = 0.0f;
    for (int r = 0; r < reps; ++r) {
        thrust::copy(source.begin(), source.end(), desc.triangles.begin());
        if (cudaDeviceSynchronize() != cudaSuccess) return -2;
        const auto w0 = std::chrono::steady_clock::now();
        cudaEventRecord(e0, 0);
        builder.build(desc, n);
        cudaEventRecord(e1, 0);
        if (cudaEventSynchronize(e1) != cudaSuccess) return -2;
        const auto w1 = std::chrono::steady_clock::now();
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        sum += ms;
        wall += std::chrono::duration<double, std::milli>(w1 - w0).count();
        least = r == 0 ? ms : std::min(least, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ms_mean) *ms_mean = (float)(sum / reps);
    if (ms_min) *ms_min = least;
    if (wall_ms_mean) *wall_ms_mean = (float)(wall / reps);
    if (tris_out) thrust::copy(desc.triangles.begin(), desc.triangles.end(), static_cast<CUDA::Triangle*>(tris_out));
    if (children_out)
        thrust::copy(desc.children.begin(), desc.children.end(), reinterpret_cast<Node*>(children_out));
    if (parents_leaf_out) thrust::copy(desc.parents[0].begin(), desc.parents[0].end(), parents_leaf_out);
    if (parents_internal_out) thrust::copy(desc.parents[1].begin(), desc.parents[1].end(), parents_internal_out);
    if (boxes_out)
        thrust::copy(desc.internalNodeBBoxes.begin(), desc.internalNodeBBoxes.end(), reinterpret_cast<BBox*>(boxes_out));
    trace("build: done");
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

// CUDAPathTracer's own methods (compiled with the kernel) refer to CUDA::Scene, whose
// upload path (Scene.cu) logs through the engine's SDL/OpenGL logger; the render entry
// below fills the same descriptors itself, so the class only needs to link.
CUDA::Scene* CUDA::Scene::m_activeScene{nullptr};
CUDA::Scene::Scene() {}
CUDA::Scene::~Scene() {}
void CUDA::Scene::upload(const CUDA::HostSceneDescription&) {}
PathTracerSettings::Demo PathTracerSettings::DEMO;
PathTracerSettings::GISettings PathTracerSettings::GI;

static int refgpu_render_impl(const void* tris_host, uint32_t n, const float* box, const void* infos_host,
                              uint32_t info_count, uint32_t width, uint32_t height, const float* cam15,
                              uint32_t bounces, float intensity, int stratified, uint32_t warmup, uint32_t frames,
                              uint32_t seed, float* ms_per_frame, float* build_ms, float* image_out)
{
    if (!tris_host || !box || !infos_host || !cam15 || n < 2 || width < 8 || height < 8 || frames < 1 ||
        bounces > 255)
        return -1;
    trace("render: start");
    StdoutToStderr quiet;
    const CUDA::Triangle* in = static_cast<const CUDA::Triangle*>(tris_host);
    const CUDA::TriangleInfo* inf = static_cast<const CUDA::TriangleInfo*>(infos_host);
    // Scene::upload (Scene.cu:28-55): triangles and shading records to the device, the
    // LBVH build, the four descriptors
    CUDA::DeviceSceneDescription desc;
    desc.triangles.assign(in, in + n);
    desc.triangleInfo.assign(inf, inf + info_count);
    desc.enclosingBBox = BBox(glm::vec3(box[0], box[1], box[2]), glm::vec3(box[3], box[4], box[5]));
    trace_error("render: scene uploaded");
    CUDA::BVHBuilder builder;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -2;
    cudaEventRecord(e0, 0);
    builder.build(desc, n);
    cudaEventRecord(e1, 0);
    if (const cudaError_t e = cudaEventSynchronize(e1)) return fail(e, "render: build");
    if (build_ms) cudaEventElapsedTime(build_ms, e0, e1);
    trace_error("render: built");
    GeometryData geometry(thrust::raw_pointer_cast(desc.internalNodeBBoxes.data()),
                          thrust::raw_pointer_cast(desc.children.data()),
                          thrust::raw_pointer_cast(desc.triangles.data()), n);
    ShadingData shading(thrust::raw_pointer_cast(desc.triangleInfo.data()));
    shading.textures = nullptr;  // untextured materials (albedo / normal-map indices are invalid)
    LightingData lighting;
    lighting.dirLightCount = 0;  // the benchmark's light is an emissive quad
    lighting.dirLights = nullptr;
    lighting.indirectIntensity = intensity;
    lighting.indirectBounceCount = static_cast<uint8_t>(bounces);
    MiscData misc;
    misc.useStratifiedSampling = stratified != 0;
    const cudaError_t copied[4] = {cudaMemcpyToSymbol(g_geometryData, &geometry, sizeof(geometry)),
                                   cudaMemcpyToSymbol(g_shadingData, &shading, sizeof(shading)),
                                   cudaMemcpyToSymbol(g_lightingData, &lighting, sizeof(lighting)),
                                   cudaMemcpyToSymbol(g_miscData, &misc, sizeof(misc))};
    for (int k = 0; k < 4; ++k)
        if (copied[k] != cudaSuccess) return fail(copied[k], "render: scene descriptor copy");
    trace_error("render: descriptors set");
    // the screen texture: a float4 array with surface load/store, cleared (frame 0's
    // running mean reads it: lerp(hit, old, 0))
    cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
    cudaArray_t screen = nullptr;
    if (const cudaError_t e = cudaMallocArray(&screen, &ch, width, height, cudaArraySurfaceLoadStore))
        return fail(e, "render: screen array");
    std::vector<float> zeros((size_t)width * height * 4, 0.0f);
    cudaMemcpy2DToArray(screen, 0, 0, zeros.data(), width * sizeof(float4), width * sizeof(float4), height,
                        cudaMemcpyHostToDevice);
    cudaResourceDesc res;
    memset(&res, 0, sizeof(res));
    res.resType = cudaResourceTypeArray;
    res.res.array.array = screen;
    cudaSurfaceObject_t surf = 0;
    if (const cudaError_t e = cudaCreateSurfaceObject(&surf, &res)) {
        cudaFreeArray(screen);
        return fail(e, "render: surface object");
    }
    trace_error("render: surface created");
    const glm::vec3 eye(cam15[0], cam15[1], cam15[2]);
    const glm::vec3 d00(cam15[3], cam15[4], cam15[5]), d10(cam15[6], cam15[7], cam15[8]);
    const glm::vec3 d11(cam15[9], cam15[10], cam15[11]), d01(cam15[12], cam15[13], cam15[14]);
    // CUDAPathTracer::raytrace (cuda_path_tracer.cu:444-459): 8x8 blocks over the
    // truncated grid, one sample per launch, a new random seed per frame
    const dim3 threads(8, 8), blocks(width / 8, height / 8);
    Random::seed(seed);
    uint32_t frame = 0;
    for (uint32_t f = 0; f < warmup; ++f, ++frame)
        raytrace_kernel<<<blocks, threads>>>(surf, eye, d00, d10, d11, d01, glm::ivec2(width, height), frame,
                                             Random::getUInt(0, std::numeric_limits<uint32_t>().max()));
    trace_error("render: warm-up launched");
    if (const cudaError_t e = cudaDeviceSynchronize()) {
        cudaDestroySurfaceObject(surf);
        cudaFreeArray(screen);
        return fail(e, "render: warm-up frames");
    }
    trace_error("render: warm-up done");
    cudaEventRecord(e0, 0);
    for (uint32_t f = 0; f < frames; ++f, ++frame)
        raytrace_kernel<<<blocks, threads>>>(surf, eye, d00, d10, d11, d01, glm::ivec2(width, height), frame,
                                             Random::getUInt(0, std::numeric_limits<uint32_t>().max()));
    cudaEventRecord(e1, 0);
    trace_error("render: frames launched");
    const cudaError_t err = cudaEventSynchronize(e1);
    trace_error("render: frames done");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms_per_frame) *ms_per_frame = ms / frames;
    if (err == cudaSuccess && image_out)
        cudaMemcpy2DFromArray(image_out, width * sizeof(float4), screen, 0, 0, width * sizeof(float4), height,
                              cudaMemcpyDeviceToHost);
    cudaDestroySurfaceObject(surf);
    cudaFreeArray(screen);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // release the vectors here, where a failure is still caught by the caller's handler
    // (their destructors would run destroy kernels where an exception cannot propagate)
    release(desc.triangles);
    release(desc.triangleInfo);
    release(desc.children);
    release(desc.parents[0]);
    release(desc.parents[1]);
    release(desc.internalNodeBBoxes);
    trace_error("render: released");
    return err == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : -2;
}

extern "C" {

// The reference's renderer on this GPU: Scene::upload's work (its LBVH build, timed
// into *build_ms) for n triangles with info_count shading records, then `warmup`
// untimed and `frames` timed launches of raytrace_kernel at width x height (one sample
// per pixel per launch, the running mean in a float4 surface), the camera as eye and
// four corner directions (00, 10, 11, 01), `bounces` indirect bounces, no directional
// lights. *ms_per_frame: mean device time of a timed launch. image_out (nullable,
// width x height x 4 floats): the running-mean image after the last frame. Returns 0,
// -1 for bad arguments, -2 for a CUDA error, -3 when thrust threw.
REFGPU_API int refgpu_render(const void* tris_host, uint32_t n, const float* box, const void* infos_host,
                             uint32_t info_count, uint32_t width, uint32_t height, const float* cam15, uint32_t bounces,
                             float intensity, int stratified, uint32_t warmup, uint32_t frames, uint32_t seed,
                             float* ms_per_frame, float* build_ms, float* image_out)
{
    try {
        return refgpu_render_impl(tris_host, n, box, infos_host, info_count, width, height, cam15, bounces, intensity,
                                  stratified, warmup, frames, seed, ms_per_frame, build_ms, image_out);
    } catch (const std::exception& e) {
        fprintf(stderr, "refgpu_render: %s\n", e.what());
    } catch (...) {
        fprintf(stderr, "refgpu_render: unknown exception\n");
    }
    return -3;
}

}  // extern "C"
