// LBVH build for callers that cannot allocate device memory (cpt_lbvh_build_static).
//
// Some hosts of this library cannot call cudaMalloc when they want a BVH: an engine
// plugin whose host application owns every device allocation and hands the plugin
// only its input and output buffers; a real-time frame loop that must not allocate
// (cudaMalloc and cudaFree can synchronize the device and stall the frame); code
// running under a fixed, pre-reserved device-memory budget. For them the build's
// scratch lives in a fixed array in the library's own device image instead of a
// caller allocation. The array is created when the library's device code is loaded
// on a GPU, and every GPU that loads the library holds it until the process exits.
#include <cuda_runtime.h>
#include <mutex>
#include "cpt.h"
#include "cpt_internal.h"

namespace {

constexpr size_t kStaticScratchBytes = CPT_LBVH_STATIC_SCRATCH_BYTES;
constexpr uint32_t kStaticMaxTriangles = CPT_LBVH_STATIC_MAX_TRIANGLES;

// The shared scratch. In host code this name is only a host-side stand-in for
// the device symbol, never a device address: the address a kernel may use comes
// from cudaGetSymbolAddress, taken per device below.
static __device__ __align__(256) unsigned char g_lbvh_static_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device; looked up once per
// device (with that device current) and cached for the life of the process, so the
// lookup never runs inside a stream capture after the first call. A device reset
// (cudaDeviceReset, or a destroyed and recreated primary context) reloads the device
// image and leaves the cached address stale; the header tells callers so.
int scratch_address(void** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return CPT_ERR_NO_DEVICE;
    if (dev >= kMaxDevices) return CPT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_lbvh_static_scratch) != cudaSuccess || !p) return CPT_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CPT_OK;
}

}  // namespace

extern "C" int cpt_lbvh_build_static(const cpt_triangle* tris_in, uint32_t n, const float* enclosing_box,
                                     int morton_bits, cpt_bvh* bvh, uint32_t flags, cudaStream_t stream)
{
    CPT_RANGE("cpt_lbvh_build_static");
    if (n > kStaticMaxTriangles) return CPT_ERR_SCRATCH_TOO_SMALL;
    if (n < 2 || (morton_bits != 30 && morton_bits != 63) || !tris_in || !bvh) return CPT_ERR_INVALID_ARGUMENT;
    if (cpt_lbvh_scratch_bytes(n, morton_bits) > kStaticScratchBytes) return CPT_ERR_SCRATCH_TOO_SMALL;
    void* scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != CPT_OK) return rc;
    // Same build as cpt_lbvh_build; everything the build needs at zero it zeroes
    // itself on the stream (histograms, look-back words, refit counters, status).
    return cpt_lbvh_build(tris_in, n, enclosing_box, morton_bits, bvh, scratch, kStaticScratchBytes, flags, stream);
}
