// Force-included header (g++ -include) that lets the reference's CUDA sources for
// the LBVH builder and the closest-hit traversal compile as plain host C++ with
// thrust's OpenMP device system. Test infrastructure only: the product never
// links against anything built with it.
//
// What it supplies, and why:
//  * <cuda_runtime.h> first, so that __device__/__host__/__constant__ expand to
//    host attributes for g++;
//  * the standard headers the reference relies on implicitly (MSVC pulled them in
//    transitively): <initializer_list>, <cfloat>, <limits>, <algorithm>, <iostream>;
//  * unqualified min/max on scalars (used by BVHBuilder.cu:166,171,183);
//  * __clz/__clzll (CUDA intrinsics) with CUDA's value at zero (32/64);
//  * atomicAdd on int through the GCC builtin (the refit is run sequentially
//    or under OpenMP by thrust's OMP backend);
//  * cudaMalloc/cudaMemcpy/cudaFree redirected to host memory (the builder
//    stages a 2-pointer array with them, BVHBuilder.cu:238-242,266).
#pragma once
#include <cuda_runtime.h>
#include <initializer_list>
#include <cfloat>
#include <climits>
#include <limits>
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cassert>
#include <iostream>
#include <thrust/host_vector.h>

using std::min;
using std::max;

static inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz((unsigned)x); }
static inline int __clzll(long long x) { return x == 0 ? 64 : __builtin_clzll((unsigned long long)x); }

static inline int atomicAdd(int* addr, int v) { return __atomic_fetch_add(addr, v, __ATOMIC_SEQ_CST); }

static inline cudaError_t cpt_shim_malloc(void** p, size_t n) { *p = std::malloc(n); return cudaSuccess; }
static inline cudaError_t cpt_shim_memcpy(void* d, const void* s, size_t n, int) { std::memcpy(d, s, n); return cudaSuccess; }
static inline cudaError_t cpt_shim_free(void* p) { std::free(p); return cudaSuccess; }
#define cudaMalloc(p, n) cpt_shim_malloc((void**)(p), (n))
#define cudaMemcpy(d, s, n, k) cpt_shim_memcpy((d), (s), (n), (int)(k))
#define cudaFree(p) cpt_shim_free((p))
