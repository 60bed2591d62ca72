// Emitter table for next-event estimation (cpt_emitters_build).
//
// Lists the emissive triangles of a built BVH in sorted-triangle order with the
// distribution the renderer draws them from (proportional to area):
//   header (16 B): emitter count, total area, emitters found, overflow flag
//   per emitter (48 B): (v0, cdf) (v1 - v0, area) (v2 - v0, sorted triangle index)
//
// Listing: chunks of kChunk triangles, one block each. k_emit_count counts each
// chunk's emitters, k_emit_offsets scans the chunk counts (one block), k_emit_write
// lists every chunk's emitters at its offset in triangle order. The order is that
// of the sorted triangles whatever the grid, so the table is the same every run.
//
// Distribution: area = 0.5 * |e1 x e2|. The cumulative sums are taken in segments
// of kSeg emitters: the area sums inside a segment in order (k_emit_segments), the
// segment totals in order (k_emit_total), then cdf_j = (offset of j's segment + the
// sum inside it up to j) / total (k_emit_cdf). The last emitter's cdf is exactly 1
// (its numerator is the total, summed the same way), so a uniform u in [0, 1)
// always finds an emitter with u < cdf.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include "cpt.h"
#include "cpt_device.cuh"
#include "cpt_internal.h"

namespace cpt {
namespace {

constexpr int kEmitBlock = 256;
constexpr int kEmitPerThread = 16;
constexpr uint32_t kChunk = kEmitBlock * kEmitPerThread;
constexpr uint32_t kSeg = 256;
constexpr int kScanBlock = 1024;

struct EmitterLayout {
    float4* header;
    float4* records;
    uint32_t* chunk_counts;
    uint32_t* chunk_offsets;
    float* seg_totals;
    float* seg_offsets;
    uint32_t chunks, segments;
};

inline uint32_t chunk_count(uint32_t n) { return (uint32_t)(((uint64_t)n + kChunk - 1) / kChunk); }
inline uint32_t segment_count(uint32_t cap) { return (uint32_t)(((uint64_t)cap + kSeg - 1) / kSeg); }

size_t emitter_layout(uint32_t n, uint32_t cap, void* base, EmitterLayout* out)
{
    Carver c(base);
    EmitterLayout l;
    l.chunks = chunk_count(n);
    l.segments = std::max(1u, segment_count(cap));
    l.header = c.take<float4>(1 + 3ull * cap);
    l.records = l.header + 1;
    l.chunk_counts = c.take<uint32_t>(l.chunks);
    l.chunk_offsets = c.take<uint32_t>(l.chunks);
    l.seg_totals = c.take<float>(l.segments);
    l.seg_offsets = c.take<float>(l.segments);
    if (out) *out = l;
    return c.used();
}

__device__ __forceinline__ bool is_emitter(const cpt_triangle* __restrict__ tris, uint32_t i,
                                           const cpt_triangle_info* __restrict__ infos, uint32_t info_count)
{
    const uint32_t ii = __ldg(&tris[i].info_idx);
    if (ii >= info_count) return false;
    const float* e = infos[ii].material.emission;
    return __fadd_rn(__fadd_rn(__ldg(e), __ldg(e + 1)), __ldg(e + 2)) > 1e-7f;
}

// Inclusive sum over the block of one value per thread (kEmitBlock threads).
__device__ __forceinline__ uint32_t block_inclusive_sum(uint32_t x, uint32_t* s_warp, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        const uint32_t t = s_warp[w];
        if (w < warp) before += t;
        total += t;
    }
    __syncthreads();
    return before + x;
}

__global__ void __launch_bounds__(kEmitBlock) k_emit_count(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                           const cpt_triangle_info* __restrict__ infos,
                                                           uint32_t info_count, uint32_t* __restrict__ chunk_counts)
{
    __shared__ uint32_t s_warp[kEmitBlock / 32];
    const uint64_t first = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kEmitPerThread;
    uint32_t c = 0;
    for (int k = 0; k < kEmitPerThread; ++k) {
        const uint64_t i = first + k;
        if (i < n && is_emitter(tris, (uint32_t)i, infos, info_count)) ++c;
    }
    uint32_t total;
    block_inclusive_sum(c, s_warp, total);
    if (threadIdx.x == 0) chunk_counts[blockIdx.x] = total;
}

// One block: exclusive offsets of the chunk counts; the header's count words.
__global__ void __launch_bounds__(kScanBlock) k_emit_offsets(const uint32_t* __restrict__ chunk_counts, uint32_t chunks,
                                                             uint32_t* __restrict__ chunk_offsets,
                                                             float4* __restrict__ header, uint32_t cap)
{
    __shared__ uint32_t s_warp[kScanBlock / 32];
    uint32_t carry = 0;
    for (uint32_t base = 0; base < chunks; base += kScanBlock) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t x = i < chunks ? chunk_counts[i] : 0u;
        uint32_t total;
        const uint32_t incl = block_inclusive_sum(x, s_warp, total);
        if (i < chunks) chunk_offsets[i] = carry + incl - x;
        carry += total;
    }
    if (threadIdx.x == 0) {
        const bool fits = carry <= cap;
        *header = make_float4(__uint_as_float(fits ? carry : 0u), 0.f, __uint_as_float(carry),
                              __uint_as_float(fits ? 0u : 1u));
    }
}

__global__ void __launch_bounds__(kEmitBlock) k_emit_write(const cpt_triangle* __restrict__ tris, uint32_t n,
                                                           const cpt_triangle_info* __restrict__ infos,
                                                           uint32_t info_count,
                                                           const uint32_t* __restrict__ chunk_offsets,
                                                           const float4* __restrict__ header,
                                                           float4* __restrict__ records)
{
    __shared__ uint32_t s_warp[kEmitBlock / 32];
    const uint32_t count = __float_as_uint(header->x);  // 0 when the emitters did not fit
    const uint64_t first = (uint64_t)blockIdx.x * kChunk + (uint64_t)threadIdx.x * kEmitPerThread;
    uint32_t flags = 0;
    for (int k = 0; k < kEmitPerThread; ++k) {
        const uint64_t i = first + k;
        if (i < n && is_emitter(tris, (uint32_t)i, infos, info_count)) flags |= 1u << k;
    }
    uint32_t total;
    const uint32_t c = __popc(flags);
    uint32_t slot = chunk_offsets[blockIdx.x] + block_inclusive_sum(c, s_warp, total) - c;
    if (count == 0) return;
    for (int k = 0; k < kEmitPerThread; ++k) {
        if (!(flags >> k & 1u)) continue;
        const uint32_t i = (uint32_t)(first + k);
        const cpt_triangle& t = tris[i];
        const f3 v0 = ld3(t.v0), v1 = ld3(t.v1), v2 = ld3(t.v2);
        const f3 e1 = sub(v1, v0), e2 = sub(v2, v0);
        const f3 cr = cross(e1, e2);
        const float area = __fmul_rn(0.5f, __fsqrt_rn(dot(cr, cr)));
        float4* r = records + 3 * (size_t)slot;
        r[0] = make_float4(v0.x, v0.y, v0.z, 0.f);
        r[1] = make_float4(e1.x, e1.y, e1.z, area);
        r[2] = make_float4(e2.x, e2.y, e2.z, __uint_as_float(i));
        ++slot;
    }
}

// Area sum of each segment of kSeg emitters, in order.
__global__ void __launch_bounds__(256) k_emit_segments(const float4* __restrict__ header,
                                                       const float4* __restrict__ records, uint32_t segments,
                                                       float* __restrict__ seg_totals)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t count = __float_as_uint(header->x);
    if (s >= segments || (uint64_t)s * kSeg >= count) return;
    const uint64_t seg_end = (uint64_t)(s + 1) * kSeg;
    const uint32_t end = seg_end < count ? (uint32_t)seg_end : count;
    float sum = 0.f;
    for (uint32_t j = s * kSeg; j < end; ++j) sum = __fadd_rn(sum, records[3 * (size_t)j + 1].w);
    seg_totals[s] = sum;
}

// One thread: segment offsets and the total area, summed in segment order.
__global__ void k_emit_total(float4* __restrict__ header, const float* __restrict__ seg_totals,
                             float* __restrict__ seg_offsets)
{
    if (threadIdx.x != 0) return;
    const uint32_t count = __float_as_uint(header->x);
    const uint32_t segs = (uint32_t)(((uint64_t)count + kSeg - 1) / kSeg);
    float run = 0.f;
    for (uint32_t s = 0; s < segs; ++s) {
        seg_offsets[s] = run;
        run = __fadd_rn(run, seg_totals[s]);
    }
    header->y = run;
}

__global__ void __launch_bounds__(256) k_emit_cdf(const float4* __restrict__ header, float4* __restrict__ records,
                                                  uint32_t segments, const float* __restrict__ seg_offsets)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t count = __float_as_uint(header->x);
    const float total = header->y;
    if (s >= segments || (uint64_t)s * kSeg >= count) return;
    const uint64_t seg_end = (uint64_t)(s + 1) * kSeg;
    const uint32_t end = seg_end < count ? (uint32_t)seg_end : count;
    const float off = seg_offsets[s];
    float sum = 0.f;
    for (uint32_t j = s * kSeg; j < end; ++j) {
        sum = __fadd_rn(sum, records[3 * (size_t)j + 1].w);
        records[3 * (size_t)j].w = total > 0.f ? __fdiv_rn(__fadd_rn(off, sum), total) : 0.f;
    }
}

}  // namespace
}  // namespace cpt

using namespace cpt;

extern "C" size_t cpt_emitters_bytes(uint32_t n, uint32_t max_emitters)
{
    if (n == 0) return 0;
    return emitter_layout(n, max_emitters, nullptr, nullptr);
}

extern "C" int cpt_emitters_build(const cpt_bvh* bvh, const cpt_scene* scene, uint32_t max_emitters, void* table,
                                  size_t table_bytes, uint32_t* count_out, cudaStream_t stream)
{
    CPT_RANGE("cpt_emitters_build");
    if (!bvh || !scene || !table || !bvh->tris || bvh->n == 0 || !scene->infos) return CPT_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(table) & 255) return CPT_ERR_INVALID_ARGUMENT;
    if (table_bytes < cpt_emitters_bytes(bvh->n, max_emitters)) return CPT_ERR_SCRATCH_TOO_SMALL;
    EmitterLayout l;
    emitter_layout(bvh->n, max_emitters, table, &l);
    const uint32_t n = bvh->n;
    k_emit_count<<<l.chunks, kEmitBlock, 0, stream>>>(bvh->tris, n, scene->infos, scene->info_count, l.chunk_counts);
    CPT_LAUNCH_CHECK();
    k_emit_offsets<<<1, kScanBlock, 0, stream>>>(l.chunk_counts, l.chunks, l.chunk_offsets, l.header, max_emitters);
    CPT_LAUNCH_CHECK();
    k_emit_write<<<l.chunks, kEmitBlock, 0, stream>>>(bvh->tris, n, scene->infos, scene->info_count, l.chunk_offsets,
                                                      l.header, l.records);
    CPT_LAUNCH_CHECK();
    const uint32_t seg_blocks = (l.segments + 255) / 256;
    k_emit_segments<<<seg_blocks, 256, 0, stream>>>(l.header, l.records, l.segments, l.seg_totals);
    CPT_LAUNCH_CHECK();
    k_emit_total<<<1, 32, 0, stream>>>(l.header, l.seg_totals, l.seg_offsets);
    CPT_LAUNCH_CHECK();
    k_emit_cdf<<<seg_blocks, 256, 0, stream>>>(l.header, l.records, l.segments, l.seg_offsets);
    CPT_LAUNCH_CHECK();
    if (count_out) {
        uint32_t h[4];
        CPT_CUDA_TRY(cudaMemcpyAsync(h, l.header, sizeof(h), cudaMemcpyDeviceToHost, stream));
        CPT_CUDA_TRY(cudaStreamSynchronize(stream));
        *count_out = h[2];
        if (h[3]) return CPT_ERR_SCRATCH_TOO_SMALL;
    }
    return CPT_OK;
}
