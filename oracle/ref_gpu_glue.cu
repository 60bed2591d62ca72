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
#include "engine/geometry/BBox.cpp"
#include "application/cuda/BVHBuilder.cu"

#include <chrono>
#include <cstdio>
#include <unistd.h>

namespace {

// BVHBuilder::build prints the two root volumes on stdout (BVHBuilder.cu:263-264);
// the benchmark owns stdout (one JSON line), so the builder's lines go to stderr.
struct StdoutToStderr {
    int saved;
    StdoutToStderr() { std::cout.flush(); fflush(stdout); saved = dup(1); dup2(2, 1); }
    ~StdoutToStderr() { std::cout.flush(); fflush(stdout); dup2(saved, 1); close(saved); }
};

}  // namespace

extern "C" {

int refgpu_key_bits(void) { return sizeof(MortonIntType) == 8 ? 63 : 30; }

// Uploads n triangles (host, 40-B CUDA::Triangle records) and the enclosing box
// (host, min xyz, max xyz), runs one untimed warm-up build, then `reps` builds, each
// from the unsorted triangles (restoring the input order is outside the timed span).
// Per build, CUDA events on the legacy default stream (the one the builder uses)
// bracket BVHBuilder::build; the host wall time of the call is taken beside them.
// Outputs: mean and least event time (ms), mean wall time (ms); when the array
// pointers are non-null, the last build's sorted triangles, Node words, both parent
// arrays and the internal-node boxes (24 B each) are copied to host memory.
// Returns 0, -1 for bad arguments, -2 for a CUDA error.
int refgpu_build(const void* tris_host, uint32_t n, const float* box, int reps, float* ms_mean, float* ms_min,
                 float* wall_ms_mean, void* tris_out, uint32_t* children_out, uint32_t* parents_leaf_out,
                 uint32_t* parents_internal_out, float* boxes_out)
{
    if (!tris_host || !box || n < 2 || reps < 1) return -1;
    StdoutToStderr quiet;
    const CUDA::Triangle* in = static_cast<const CUDA::Triangle*>(tris_host);
    thrust::device_vector<CUDA::Triangle> source(in, in + n);
    CUDA::DeviceSceneDescription desc;
    desc.triangles = source;
    desc.enclosingBBox = BBox(glm::vec3(box[0], box[1], box[2]), glm::vec3(box[3], box[4], box[5]));
    CUDA::BVHBuilder builder;
    builder.build(desc, n);  // warm-up: first allocations, thrust's temporary storage
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
    return cudaGetLastError() == cudaSuccess ? 0 : -2;
}

}  // extern "C"
