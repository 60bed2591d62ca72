// Wavefront-render extension points used by the radiance cache and the tracer object.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>
#include "cpt.h"

namespace cpt {

// Optional per-render hook. With `records` set, every path that reaches vertex
// `record_depth` appends one record of 5 float4 (compact, in no particular order):
//   (position, path id) (ray direction, W.x) (normal, W.y) (albedo, W.z) (R, 0)
// with W = indirect_intensity x the path's throughput after that vertex's albedo and
// R its radiance so far. `after_wave` runs once per wave after the last bounce and
// before the wave's samples are accumulated; it may add to the paths' radiance
// (`state`: 2 float4 per path, radiance in the first). image_pass = false renders
// no image: no accumulation and no frame-counter advance.
//
// Training on the image's own paths (train_stride > 0): a path whose (pixel, sample)
// hash is 0 modulo train_stride is a training path — at vertex record_depth it
// appends its record to train_records (at most train_capacity per wave, counted in
// *train_count; later ones are dropped) instead of `records`, and goes on to full
// depth. With cut_at_record, every other path ends at vertex record_depth (no bounce
// ray, no shadow ray from it): its remainder is what after_wave adds.
struct RenderHook {
    float4* records;
    uint32_t capacity;  // records the buffer holds; must cover a wave
    uint32_t record_depth;
    bool image_pass;
    float4* train_records;
    uint32_t* train_count;  // device word, zeroed by the hook's owner
    uint32_t train_capacity;
    uint32_t train_stride;  // 0: no training paths
    bool cut_at_record;
    int (*after_wave)(void* ctx, const float4* records, const uint32_t* record_count, uint32_t capacity,
                      float4* state, cudaStream_t stream);
    void* ctx;
    // nullable: the first shading launch waits for this event (the shading records or
    // lights may still be on their way to the device; the traversal before it does not
    // read them)
    cudaEvent_t shade_after;
};

// Bytes of a record buffer for this render (0 on bad arguments); *capacity gets
// the records one wave can produce.
size_t render_hook_layout(const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* reserved,
                          uint32_t* capacity);

int cpt_render_views_hooked(const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* scratch,
                            size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
                            const RenderHook* hook, cudaStream_t stream);

}  // namespace cpt
