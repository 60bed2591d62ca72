// Host-side helpers shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include <nvtx3/nvToolsExt.h>
#include <atomic>
#include "cpt.h"

namespace cpt {

// An NVTX range named after the entry point, open for the call's host-side duration,
// so that profilers (Nsight Systems, Nsight Compute's --nvtx filters) group the kernels
// a call launches under it. Without a profiler attached NVTX calls do nothing.
struct Range {
    explicit Range(const char* name) { nvtxRangePushA(name); }
    ~Range() { nvtxRangePop(); }
    Range(const Range&) = delete;
    Range& operator=(const Range&) = delete;
};

// Count of kernel launches issued by this library (reported by cpt_launch_count).
extern std::atomic<unsigned long long> g_launches;
inline void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Sequential carve-out of one allocation into 256-byte aligned pieces.
struct Carver {
    char* base;
    size_t off = 0;
    explicit Carver(void* p) : base(static_cast<char*>(p)) {}
    template <typename T>
    T* take(size_t count)
    {
        off = align_up(off, 256);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
    size_t used() const { return align_up(off, 256); }
};

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? CPT_OK : CPT_ERR_CUDA; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Kernel identities for cpt_profile_*.
enum KernelId {
    K_BOUNDS, K_MORTON, K_SCAN, K_ONESWEEP, K_TOPOLOGY, K_GATHER_REFIT, K_TRACE,
    K_GENERATE, K_EXTEND, K_SHADE, K_WAVE_COUNTS, K_ACCUMULATE, K_RESOLVE, K_RAY_SORT,
    K_RC_INFER, K_RC_TRAIN, K_RC_ADAM, K_RC_COLLECT, K_OCCLUDE, K_KERNEL_COUNT
};
extern const char* const kKernelNames[K_KERNEL_COUNT];
extern std::atomic<bool> g_profiling;

// Brackets one launch with two events on its stream while profiling is on.
struct ProfScope {
    int id;
    cudaStream_t stream;
    cudaEvent_t start = nullptr;
    ProfScope(int id_, cudaStream_t s);
    ~ProfScope();
};

constexpr uint32_t kMaxTriangles = (1u << 30) - 1;  // 30-bit node indices (Node.h:13-15)

}  // namespace cpt

#define CPT_PROF_CAT2(a, b) a##b
#define CPT_PROF_CAT(a, b) CPT_PROF_CAT2(a, b)
#define CPT_PROF(id, stream) ::cpt::ProfScope CPT_PROF_CAT(prof_scope_, __LINE__)((id), (stream))
#define CPT_RANGE(name) ::cpt::Range CPT_PROF_CAT(nvtx_range_, __LINE__)(name)

#define CPT_LAUNCH_CHECK()                                          \
    do {                                                            \
        ::cpt::note_launch();                                       \
        cudaError_t e_ = cudaGetLastError();                        \
        if (e_ != cudaSuccess) return CPT_ERR_CUDA;                 \
    } while (0)

#define CPT_CUDA_TRY(expr)                                          \
    do {                                                            \
        cudaError_t e_ = (expr);                                    \
        if (e_ != cudaSuccess) return CPT_ERR_CUDA;                 \
    } while (0)
