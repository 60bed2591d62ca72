/* cpt — B200-native LBVH builder and progressive path tracer (C ABI).
 *
 * Drop-in replacement for the hot path of compix/CUDA-Path-Tracer: a triangle
 * soup goes in; the reference's BVH arrays, compact traversal nodes and an
 * accumulated framebuffer come out. All functions are plain C with device
 * pointers owned by the caller (unless a function says otherwise), an explicit
 * CUDA stream and an int status (CPT_OK = 0). Work is enqueued on the stream and
 * returns immediately unless a flag asks for a synchronous check.
 *
 * Layout structs mirror the reference byte for byte:
 *   cpt_triangle       == CUDA::Triangle       (source/application/cuda/geometry.h:20-30)
 *   cpt_bbox           == BBox                 (source/engine/geometry/BBox.h:6-53)
 *   cpt_triangle_info  == CUDA::TriangleInfo   (source/application/cuda/TriangleInfo.h:14-75)
 *   cpt_dir_light      == CUDA::DirectionalLight (source/application/cuda/Lights.h:6-11)
 *   children / parents == Node / NodeIndex     (source/application/cuda/Node.h:8-137)
 */
#ifndef CPT_H
#define CPT_H
#include <stddef.h>
#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CPT_OK 0
#define CPT_ERR_INVALID_ARGUMENT 1  /* null pointer, n < 2, bad key width, size overflow */
#define CPT_ERR_CUDA 2              /* a CUDA runtime call failed */
#define CPT_ERR_SCRATCH_TOO_SMALL 3 /* scratch_bytes below the matching *_scratch_bytes() */
#define CPT_ERR_NONFINITE_INPUT 4   /* a vertex coordinate is NaN or infinite */
#define CPT_ERR_DEVICE_TIMEOUT 5    /* a bounded device-side wait gave up (sort look-back) */
#define CPT_ERR_STACK_OVERFLOW 6    /* a ray needed more than CPT_TRAVERSAL_STACK entries */
#define CPT_ERR_CHECK_FAILED 7      /* root box volume differs from the enclosing box's */
#define CPT_ERR_NO_DEVICE 8         /* no CUDA device / library built for another arch */
#define CPT_ERR_BAD_INDEX 9         /* a device-side index was out of range (e.g. info_idx >= info_count) */
#define CPT_ERR_TREE_TOO_DEEP 10    /* a built tree is taller than CPT_TRAVERSAL_STACK (split BVH not used) */

/* device status-word bits (cpt_bvh.status[0], render status) */
#define CPT_STATUS_NONFINITE 1u
#define CPT_STATUS_TIMEOUT 2u
#define CPT_STATUS_STACK_OVERFLOW 4u
#define CPT_STATUS_BAD_INDEX 8u /* an index read from device data was out of range (corrupt input) */

#define CPT_TRAVERSAL_STACK 64 /* MAX_TRAVERSAL_STACK_SIZE, source/engine/cuda/cuda_defs.h:21 */
#define CPT_INVALID_INDEX 0xFFFFFFFFu

/* ---- reference layouts ---- */
typedef struct cpt_triangle { float v0[3], v1[3], v2[3]; uint32_t info_idx; } cpt_triangle; /* 40 B */
typedef struct cpt_bbox { float min[3], max[3]; } cpt_bbox;                                  /* 24 B */
typedef struct cpt_vertex { float color[3], uv[2], normal[3], tangent[3], bitangent[3]; } cpt_vertex; /* 56 B */
typedef struct cpt_material {
    float emission[3];
    float specularity;
    uint32_t albedo_idx;     /* index into cpt_scene.textures, or CPT_INVALID_INDEX */
    uint32_t normal_map_idx; /* idem (tangent-space normal map) */
} cpt_material;                                                                   /* 24 B */
typedef struct cpt_triangle_info { cpt_vertex vertices[3]; cpt_material material; } cpt_triangle_info; /* 192 B */
typedef struct cpt_dir_light { float color[3], direction[3], intensity; } cpt_dir_light;               /* 28 B */

/* ---- LBVH ---- */
/* Outputs of one build. Every pointer is device memory of the stated length;
 * cpt_bvh_bind() carves them all out of one caller allocation. */
typedef struct cpt_bvh {
    uint32_t n;                 /* triangles (leaves); internal nodes are n - 1 */
    int32_t morton_bits;        /* 30 (uint32 keys) or 63 (uint64 keys) */
    cpt_triangle* tris;         /* [n]   triangles in Morton order (reference: permuted in place) */
    void* keys;                 /* [n]   sorted Morton keys */
    uint32_t* children;         /* [n-1] Node words: (left << 2) | rightInternal << 1 | leftInternal */
    uint32_t* parents_leaf;     /* [n]   parent of each leaf */
    uint32_t* parents_internal; /* [n-1] parent of each internal node; [0] = CPT_INVALID_INDEX */
    cpt_bbox* node_boxes;       /* [n-1] internal node boxes */
    void* nodes;                /* [n-1] 96-B traversal nodes: two 40-B child slots, the Node word, the
                                 *       right child's index (left + 1 here) and the far end j of the
                                 *       node's leaf range [min(i, j), max(i, j)], where a slot holds the
                                 *       child's box (internal child) or the child triangle as v0, its
                                 *       index in tris, v1 - v0, v2 - v0 (leaf child) */
    uint32_t* status;           /* [4]   device status words (CPT_STATUS_* bits in [0]) */
    void* split_nodes;          /* nullable: traversal nodes of the split BVH (cpt_lbvh_split); when set,
                                 *       tracing and rendering traverse them instead of `nodes`.
                                 *       cpt_lbvh_build clears it (the split tree is of the old triangles) */
    uint32_t split_capacity;    /* pieces the split nodes were built for (0 when none) */
    void* wide_nodes;           /* nullable: compressed 8-wide nodes (cpt_lbvh_wide); when set, tracing and
                                 *       rendering traverse them. cpt_lbvh_build and cpt_lbvh_split clear it */
    void* wide_tris;            /*       and their 48-B triangle records */
    uint32_t wide_capacity;     /* leaves of the binary tree the wide tree was built from (0 when none) */
} cpt_bvh;

/* Bytes of device memory cpt_bvh_bind() needs for n triangles. */
size_t cpt_bvh_bytes(uint32_t n, int morton_bits);
/* Lays the cpt_bvh arrays out in mem (256-B aligned pieces). */
int cpt_bvh_bind(void* mem, size_t bytes, uint32_t n, int morton_bits, cpt_bvh* out);
/* Scratch bytes cpt_lbvh_build() needs (keys, sort buffers, look-back, counters). */
size_t cpt_lbvh_scratch_bytes(uint32_t n, int morton_bits);

#define CPT_BUILD_CHECK 1u /* synchronize, map device status to a code, verify the root box */
/* The sort's decoupled look-back is the build's only device-side wait; it gives up
 * after a poll limit per tile, records CPT_STATUS_TIMEOUT, and the build's later
 * kernels then return at once (the call, or cpt_status_check, reports
 * CPT_ERR_DEVICE_TIMEOUT). CPT_BUILD_LOOKBACK_LIMIT(k), k in 1..31, sets the limit to
 * 2^k polls (default 2^22, k = 0). CPT_BUILD_TEST_WITHHOLD exercises that failure
 * path without a fault: the first sort pass's first tile never publishes its digit
 * counts, so every look-back that reaches it waits out the limit; it requires an
 * explicit limit of at most 2^16 polls (else CPT_ERR_INVALID_ARGUMENT). Other flag
 * bits are refused. */
#define CPT_BUILD_TEST_WITHHOLD 2u
#define CPT_BUILD_LOOKBACK_LIMIT(k) (((uint32_t)(k) & 31u) << 8)

/* Builds the LBVH of n >= 2 triangles.
 * Replaces CUDA::BVHBuilder::build (source/application/cuda/BVHBuilder.h:15,
 * BVHBuilder.cu:207-269). tris_in may equal bvh->tris (in-place, as the
 * reference). enclosing_box is a HOST pointer to (min xyz, max xyz), as the
 * reference's DeviceSceneDescription::enclosingBBox, or NULL to compute it on
 * the device. Outputs are bit-identical to the reference's for the same inputs. */
int cpt_lbvh_build(const cpt_triangle* tris_in, uint32_t n, const float* enclosing_box, int morton_bits,
                   cpt_bvh* bvh, void* scratch, size_t scratch_bytes, uint32_t flags, cudaStream_t stream);

/* Batched LBVH build: the LBVHs of `scenes` triangle soups in one fixed sequence of
 * launches, each launch covering every scene (one Morton launch, one stable radix
 * sort over all scenes — the key digits, then a scene-id digit —, one topology launch,
 * one refit launch). Replaces `scenes` calls of CUDA::BVHBuilder::build
 * (source/application/cuda/BVHBuilder.cu:207-269), one per scene; every scene's
 * outputs are bit-identical to cpt_lbvh_build's on the same triangles and box.
 * Host arrays of `scenes` entries: tris_in[s] (device triangles; may equal
 * bvhs[s]->tris for an in-place build), n[s] >= 2, bvhs[s] (bound for n[s] and
 * morton_bits); boxes: host, 6 floats per scene (min xyz, max xyz), each scene's
 * enclosingBBox as the reference's caller computes it (cpt_scene_bounds). The total
 * triangle count must stay below 2^30. The kernels receive the scene table by value,
 * so a call can be captured in a CUDA graph. flags: CPT_BUILD_CHECK (checks every
 * scene's status and root volume; synchronizes) or 0. */
#define CPT_MAX_BATCH_SCENES 64
size_t cpt_lbvh_batch_scratch_bytes(const uint32_t* n, uint32_t scenes, int morton_bits);
int cpt_lbvh_build_batch(const cpt_triangle* const* tris_in, const uint32_t* n, uint32_t scenes, const float* boxes,
                         int morton_bits, cpt_bvh* const* bvhs, void* scratch, size_t scratch_bytes, uint32_t flags,
                         cudaStream_t stream);

/* LBVH build that allocates nothing: the same build and outputs as
 * cpt_lbvh_build, with its scratch in a fixed array inside the library's device
 * image instead of a caller buffer. It has no counterpart in the reference, whose
 * builder resizes thrust vectors and cudaMallocs on every build
 * (BVHBuilder.cu:220-242). It is for callers that cannot allocate device memory
 * when they build: a plugin whose host application owns all device allocations,
 * a frame loop that must not allocate (allocation can synchronize the device), a
 * fixed memory budget. The caller still owns tris_in and every bvh output array.
 * Limits and rules:
 *  - n <= CPT_LBVH_STATIC_MAX_TRIANGLES (131,072); larger n returns
 *    CPT_ERR_SCRATCH_TOO_SMALL before any device work;
 *  - the array (CPT_LBVH_STATIC_SCRATCH_BYTES, 8 MiB) is created on every GPU
 *    that loads the library and held until the process exits;
 *  - the first call on a device looks up the array's device address with that
 *    device current (cudaGetSymbolAddress) — make that first call before any
 *    stream capture. The address is kept for the life of the process: after a
 *    cudaDeviceReset (or anything else that destroys and recreates the device's
 *    primary context) the library's device image is loaded anew and the kept
 *    address is stale, so do not call this entry point on that device again;
 *  - all calls share the one array: calls whose work overlaps on a GPU (e.g. on
 *    two streams) race; serialize them. Each call zeroes what must start at zero,
 *    so leftovers of the previous call are harmless. */
#define CPT_LBVH_STATIC_MAX_TRIANGLES 131072u
#define CPT_LBVH_STATIC_SCRATCH_BYTES (8u << 20)
int cpt_lbvh_build_static(const cpt_triangle* tris_in, uint32_t n, const float* enclosing_box, int morton_bits,
                          cpt_bvh* bvh, uint32_t flags, cudaStream_t stream);

/* Split traversal BVH (no reference counterpart; an optional traversal accelerator).
 * Built from an LBVH's Morton-sorted triangles: triangles whose box is large for
 * their area (long thin ones) are cut into up to 64 pieces along their longest box
 * axis, each piece keeping the box of the triangle clipped to its slab (widened by
 * 2^-20 of the coordinates so rounding cannot lose a hit); the pieces get their
 * own LBVH (Morton keys of the piece box centres in the root box, the same sort,
 * topology and refit kernels). The extra pieces are shared out in proportion to
 * sqrt(box area - 2 x triangle area), at most extra_ratio x n of them. Leaves hold
 * the whole triangle and its sorted index, so tracing reports the same triangles
 * (t, u, v and index) as over `nodes`, except that of two triangles hit at exactly
 * the same t either may be reported. The reference-format outputs are not touched.
 * Sets bvh->split_nodes = nodes and bvh->split_capacity. node_bytes / scratch bytes
 * from cpt_lbvh_split_bytes (0 on bad arguments); scratch is free after the stream
 * passes the call. */
#define CPT_SPLIT_TREELET 2u /* treelet restructuring of the Karras topology (treelets of up to 7 leaves, least
                               * total node surface area, never taller; Karras and Aila 2013 — the optimisation
                               * the reference's README cites): fewer node visits, longer build. Other flag
                               * bits are refused (CPT_ERR_INVALID_ARGUMENT; 0 from cpt_lbvh_split_bytes) */
size_t cpt_lbvh_split_bytes(uint32_t n, int morton_bits, float extra_ratio, uint32_t flags, size_t* node_bytes);
int cpt_lbvh_split(cpt_bvh* bvh, float extra_ratio, uint32_t flags, void* nodes, size_t node_bytes, void* scratch,
                   size_t scratch_bytes, cudaStream_t stream);

/* Reads the device status words of a build or render (synchronizes the stream)
 * and maps them to a status code. */
int cpt_status_check(const uint32_t* d_status, cudaStream_t stream);

/* ---- traversal ---- */
typedef struct cpt_hit { float t, u, v; uint32_t tri; } cpt_hit; /* t = FLT_MAX, tri = CPT_INVALID_INDEX on miss */

/* Closest hit (any_hit = 0) or occlusion (any_hit = 1) for n rays.
 * Replaces CUDA::trace / CUDA::shadowRay (source/application/cuda/trace.h:45-50,73-169).
 * rays: n x 8 floats (origin xyz, unused, direction xyz, unused), device. As in the
 * reference there is no ray interval: a hit counts at any t >= 0, with no far limit
 * (intersection.h:58); the unused words are ignored.
 * stats (nullable, device): n x 2 uint32 — internal nodes fetched, triangle tests. */
int cpt_trace(const cpt_bvh* bvh, const float* rays, uint32_t n, int any_hit, cpt_hit* hits, uint32_t* stats,
              cudaStream_t stream);

/* ---- path tracer ---- */
typedef struct cpt_scene {
    const cpt_triangle_info* infos; /* device, indexed by cpt_triangle.info_idx */
    uint32_t info_count;
    const cpt_dir_light* lights;    /* device */
    uint32_t light_count;
    const cudaTextureObject_t* textures; /* device array of texture handles (cpt_texture_create), nullable */
    uint32_t texture_count;
    const void* emitters;           /* device, nullable: emitter table (cpt_emitters_build) of this scene's
                                     * BVH, read when cpt_render_params.nee is set */
} cpt_scene;

/* A 2D texture for albedo / normal maps: RGBA8 texels (host memory, row-major),
 * sampled like the reference's textures (Scene.cu:57-81): normalized coordinates,
 * bilinear filtering, wrap addressing, values read as floats in [0, 1]. The
 * reference samples its mipmapped arrays with tex2D, i.e. level 0, which is what
 * this single-level texture holds. */
int cpt_texture_create(const uint8_t* rgba8, uint32_t width, uint32_t height, cudaTextureObject_t* out);
void cpt_texture_destroy(cudaTextureObject_t tex);
/* tex2D<float4>(tex, u, v) for n coordinate pairs (device uv[2n] -> device rgba_out[4n]):
 * the sampler the shader reads, exposed for parity tests. No reference counterpart. */
int cpt_texture_sample(cudaTextureObject_t tex, const float* uv, uint32_t n, float* rgba_out, cudaStream_t stream);

/* Eye and the four corner ray directions (00, 10, 11, 01) of
 * CUDAPathTracer::setPrimaryRays/setEyePos (cuda_path_tracer.h:19-21). With
 * jitter = 1 the corner directions are re-derived per sample from
 * inv_view_proj (column-major) with an NDC offset of up to +-jitter_x/y, the
 * per-frame jitter of PathTracingApp::screenToRay (PathTracingApp.cpp:217-242). */
typedef struct cpt_camera {
    float eye[3];
    float dirs[4][3];
    float inv_view_proj[16];
    float jitter_x, jitter_y;
    uint32_t jitter;
} cpt_camera;

#define CPT_ACCUM_KAHAN 0u /* float4 sum (w = samples) + float4 compensation per pixel */
#define CPT_ACCUM_LERP 1u  /* reference running mean: float4 per pixel (cuda_path_tracer.cu:413-420) */
#define CPT_ACCUM_F64 2u   /* double4 sum (w = samples) per pixel, for the RMSE reference image */

typedef struct cpt_render_params {
    uint32_t width, height;
    uint32_t spp;              /* samples rendered by this call */
    uint32_t frame0;           /* global sample index of the first (reference frame number) */
    uint32_t bounces;          /* indirectBounceCount (depth - 1) */
    float indirect_intensity;  /* indirectIntensity */
    uint32_t stratified;       /* useStratifiedSampling */
    uint32_t seed_lo, seed_hi; /* Philox key */
    uint32_t accum_mode;       /* CPT_ACCUM_* */
    uint32_t ref_grid;         /* 1: render only the reference's (W/8*8) x (H/8*8) grid */
    uint32_t wave_paths;       /* paths in flight per wave (0: library default) */
    uint32_t trace_stats;      /* 1: count node fetches / triangle tests of extension rays (slower) */
    uint32_t ray_sort;         /* 1: sort each bounce queue by direction octant + origin Morton code
                                *    before tracing it (coherence; results are unchanged) */
    uint32_t cameras;          /* cameras rendered in one call (0 or 1: one; at most CPT_MAX_VIEWS): `camera`
                                * points to that many cpt_camera, `accum` to that many consecutive accumulators
                                * of cpt_accum_bytes() each; camera c draws from the Philox counter word 3 = c */
    uint32_t* frame_counter;   /* device, nullable: when set, the call renders global samples
                                * *frame_counter + frame0 ... and adds spp to *frame_counter at its end, so a
                                * call captured once in a CUDA graph renders the next samples on each replay */
    uint32_t nee;              /* 1: next-event estimation (see cpt_emitters_build); every view's scene needs
                                * an emitter table. 0: the reference's estimator */
    /* launch shape of the persistent traversal kernels (results are unchanged; for tuning):
     * refill_lanes: a warp takes new rays once fewer than this many of its lanes still trace
     * (1..32; 0: 31 over wide trees, 16 over binary trees); traverse_blocks_per_sm: resident
     * blocks per SM of the closest-hit traversal, at most its occupancy (0: occupancy) */
    uint32_t refill_lanes;
    uint32_t traverse_blocks_per_sm;
    /* wave_lanes: 2 splits each wave's paths into two halves traced and shaded at once on
     * the caller's stream and a second stream the library owns, the second half one
     * launch behind, so that each launch's slowest rays overlap the other half's work
     * (images unchanged); 1: one sequence on the caller's stream; 0: the library's
     * default (1). Calls with a radiance cache or ray sorting use one lane. */
    uint32_t wave_lanes;
} cpt_render_params;

size_t cpt_accum_bytes(uint32_t width, uint32_t height, uint32_t accum_mode); /* per camera / view */
size_t cpt_render_scratch_bytes(const cpt_render_params* params);

/* Renders params->spp samples into accum. Replaces CUDAPathTracer::raytrace
 * (cuda_path_tracer.cu:423-464) and raytrace_kernel (:385-421).
 * ray_counts (device, nullable): CPT_RAY_COUNTS x uint64, incremented by
 * [0] primary, [1] extension, [2] shadow rays traced, — with params->trace_stats —
 * [3] internal nodes fetched and [4] triangles tested by the closest-hit (primary +
 * extension) rays, and [8 + b] closest-hit rays traced at path depth b (b < 64).
 * status (device, nullable): CPT_STATUS_* bits are OR-ed in. */
#define CPT_RAY_COUNTS 72
int cpt_render(const cpt_bvh* bvh, const cpt_scene* scene, const cpt_camera* camera, const cpt_render_params* params,
               void* accum, void* scratch, size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status,
               cudaStream_t stream);

/* ---- batched views: several scenes and/or cameras in the same waves ----
 * A view is one image: a BVH, its shading inputs, a camera, a resolution and an
 * accumulator (device, cpt_accum_bytes(width, height, params->accum_mode)).
 * One call renders params->spp samples of up to CPT_MAX_VIEWS views; the rays of
 * all views share every wavefront launch, and a frame is a fixed sequence of
 * kernel launches on `stream` (capturable in a CUDA graph). View i draws from
 * Philox counter word 3 = i. params->width/height/cameras are not used here. */
#define CPT_MAX_VIEWS 64
typedef struct cpt_view {
    const cpt_bvh* bvh;
    const cpt_scene* scene;
    cpt_camera camera;
    uint32_t width, height;
    void* accum;
} cpt_view;
size_t cpt_render_views_scratch_bytes(const cpt_view* views, uint32_t n_views, const cpt_render_params* params);
int cpt_render_views(const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* scratch,
                     size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status, cudaStream_t stream);

/* ---- compressed 8-wide traversal BVH (an extension; no reference counterpart) ----
 * Collapses the binary traversal tree in use (the split tree when one was built,
 * else the LBVH's nodes) into 8-wide nodes of 80 B with 8-bit child boxes and
 * direction-ordered slots (a binary subtree of two leaves becomes one slot), and
 * copies the leaf triangles into 48-B records in visiting order (two record positions
 * per binary leaf are reserved). Tracing and rendering then traverse it.
 * Hits are those of the binary tree (same triangle arithmetic) up to which of several
 * exactly equal distances is reported. `leaves` for the sizes: bvh->n, or
 * bvh->split_capacity after cpt_lbvh_split. status[2] / status[3] receive the wide
 * node count and the record positions used. */
#define CPT_WIDE_SAH 1u /* choose each wide node's children by a surface-area cost computed bottom-up over
                          the binary tree (a second pass before the collapse, more scratch) instead of
                          opening the largest child: a slower build for a faster traversal */
size_t cpt_lbvh_wide_bytes(uint32_t leaves, uint32_t flags, size_t* node_bytes,
                           size_t* tri_bytes); /* returns scratch bytes */
int cpt_lbvh_wide(cpt_bvh* bvh, uint32_t flags, void* nodes, size_t node_bytes, void* tris, size_t tri_bytes,
                  void* scratch, size_t scratch_bytes, cudaStream_t stream);
/* The wide trees of `trees` (1..CPT_MAX_BATCH_SCENES) built binary trees in one fixed
 * launch sequence — one cooperative launch walks the levels of all of them — instead of
 * `trees` cpt_lbvh_wide calls (the largest-child collapse, flags 0): for many small
 * scenes rebuilt every frame. Host arrays of `trees` entries: bvhs, and each tree's node
 * and record buffers with their sizes (as cpt_lbvh_wide_bytes gives for that tree);
 * leaves[i] for the scratch size as for cpt_lbvh_wide. The kernels receive the tree
 * table by value, so a call can be captured in a CUDA graph. Each tree's wide tree is the
 * one cpt_lbvh_wide builds from it (node and record counts in its status[2] / status[3];
 * only where nodes are placed in its arrays may differ). */
size_t cpt_lbvh_wide_batch_scratch_bytes(const uint32_t* leaves, uint32_t trees);
int cpt_lbvh_wide_batch(cpt_bvh* const* bvhs, uint32_t trees, void* const* nodes, const size_t* node_bytes,
                        void* const* tris, const size_t* tri_bytes, void* scratch, size_t scratch_bytes,
                        cudaStream_t stream);

/* ---- next-event estimation (an extension; no reference counterpart) ----
 * The reference gathers emitted light only where a bounce ray happens to hit an
 * emissive triangle (blinnPhongShadingPathTrace, cuda_path_tracer.cu:303-312), so a
 * small light makes every sample a lottery. With cpt_render_params.nee = 1, every
 * vertex that bounces also draws one point on the scene's emitters (a triangle by
 * area, then a uniform point on it) and traces a shadow ray to it; emission hit by a
 * bounce ray is then left out (the camera ray still sees it). The estimate has the
 * expectation of the reference's estimator: the light the bounce would have picked
 * up by chance, e * max(-w . n_e, 0) per hit, is integrated over the emitters'
 * area instead, weighted by the cosine-sampling density cos(theta) / pi of the
 * bounce it replaces.
 *
 * The emitter table lists the emissive triangles (emission r + g + b > 1e-7, the
 * renderer's test) of a built BVH in sorted-triangle order:
 *   16-B header: emitter count (u32), total area (f32), emitters found (u32),
 *                1 when they did not fit (u32; the count is then 0)
 *   48 B per emitter: (v0, cdf) (v1 - v0, area) (v2 - v0, sorted triangle index)
 * It describes the triangles' current positions: build it again after every
 * cpt_lbvh_build of the scene (the sorted order and the vertices change). */
size_t cpt_emitters_bytes(uint32_t n, uint32_t max_emitters); /* n = bvh->n */
/* count_out (host, nullable): when set, the call synchronizes the stream, stores
 * the number of emissive triangles and returns CPT_ERR_SCRATCH_TOO_SMALL if they
 * are more than max_emitters. */
int cpt_emitters_build(const cpt_bvh* bvh, const cpt_scene* scene, uint32_t max_emitters, void* table,
                       size_t table_bytes, uint32_t* count_out, cudaStream_t stream);

/* Writes the displayable image (float4 rgba per pixel, alpha 1) of an accumulator. */
int cpt_resolve(const void* accum, uint32_t width, uint32_t height, uint32_t accum_mode, float* rgba,
                cudaStream_t stream);

/* BVH heat map: per pixel, the number of internal-node boxes the camera's primary
 * ray hits, as base_color added once per box. Replaces CUDA::computeBVHColor
 * (source/application/cuda/visualization.h:19-66). rgba: device float4 per pixel;
 * node_counts (device, nullable): the counts. base_color is a host pointer. */
int cpt_bvh_heatmap(const cpt_bvh* bvh, const cpt_camera* camera, uint32_t width, uint32_t height,
                    const float base_color[3], float* rgba, uint32_t* node_counts, cudaStream_t stream);

/* ---- reference-facing tracer object (host buffers in, image out) ----
 * Mirrors CUDAPathTracer (source/application/cuda/cuda_path_tracer.h:13-40):
 * upload a HostSceneDescription, set primary rays and eye, raytrace frame by
 * frame, reset. Owns its device memory and stream.
 * Device: the tracer belongs to the device current at cpt_tracer_create and does not
 * switch devices itself; make that device current before each call on it (one tracer
 * per GPU, as the reference's single-device application has one).
 * Host buffers: cpt_tracer_upload copies asynchronously. Pageable host memory may be
 * reused when the call returns. Page-locked (pinned) memory — which lets the copies
 * overlap the builds and earlier frames — must stay unchanged until the copies have run:
 * until cpt_tracer_read_image or cpt_tracer_ray_counts returns after a
 * cpt_tracer_raytrace of that scene. */
typedef struct cpt_tracer cpt_tracer;
int cpt_tracer_create(cpt_tracer** out, int morton_bits);
void cpt_tracer_destroy(cpt_tracer* t);
/* CUDAPathTracer::upload + Scene::upload (cuda_path_tracer.cu:466-470, Scene.cu:28-55):
 * host triangles / infos / lights, host enclosing box (NULL: computed).
 * The tracer keeps two scenes: an upload fills the one the queued frames do not read
 * (waiting on the device, not the host, for the last frame that read it), on streams of
 * its own, and the next raytrace renders it; so an upload issued while a frame is still
 * in flight (before its read-back) copies and builds beside that frame. The second
 * scene's memory is allocated at the second upload. A failed upload leaves no scene to
 * render. */
int cpt_tracer_upload(cpt_tracer* t, const cpt_triangle* tris, uint32_t n, const cpt_triangle_info* infos,
                      uint32_t info_count, const cpt_dir_light* lights, uint32_t light_count,
                      const float* enclosing_box);
/* Scene::upload(textureArrays) (Scene.cu:57-81): the texture table that
 * albedo_idx / normal_map_idx index (handles from cpt_texture_create; the caller
 * keeps them alive while the tracer renders). count 0 clears it. */
int cpt_tracer_upload_textures(cpt_tracer* t, const cudaTextureObject_t* textures, uint32_t count);
/* extra_ratio > 0: every later upload also builds the split traversal BVH
 * (cpt_lbvh_split with `flags`) and renders through it; 0 (default) renders over the LBVH. */
int cpt_tracer_set_split(cpt_tracer* t, float extra_ratio, uint32_t flags);
/* on = 1: every later upload also builds the compressed wide tree (cpt_lbvh_wide) of
 * the traversal tree (after the split tree, when one is set) and renders through it;
 * on = 2: the same with the surface-area collapse (CPT_WIDE_SAH: a longer build, a
 * faster render; for scenes uploaded once and rendered many times). 0: off. */
int cpt_tracer_set_wide(cpt_tracer* t, uint32_t on);
/* on = 1: render with next-event estimation (cpt_render_params.nee); the tracer
 * builds the uploaded scene's emitter table on the next raytrace. Switching
 * restarts the accumulation (frame 0). Default 0: the reference's estimator. */
int cpt_tracer_set_nee(cpt_tracer* t, uint32_t on);
int cpt_tracer_set_primary_rays(cpt_tracer* t, const float dirs[12]);
int cpt_tracer_set_eye(cpt_tracer* t, const float eye[3]);
int cpt_tracer_set_camera(cpt_tracer* t, const cpt_camera* cam);
/* GI settings (PathTracingSettings.h:26-28) and the seed of the random stream. */
int cpt_tracer_set_settings(cpt_tracer* t, uint32_t bounces, float indirect_intensity, uint32_t stratified,
                            uint32_t seed_lo, uint32_t seed_hi, uint32_t accum_mode);
/* Renders spp samples (frames) at width x height; the frame counter advances by spp. */
int cpt_tracer_raytrace(cpt_tracer* t, uint32_t width, uint32_t height, uint32_t spp);
void cpt_tracer_reset_frames(cpt_tracer* t);
uint32_t cpt_tracer_frame(const cpt_tracer* t);
/* Copies the resolved image (float4 per pixel) to host memory; synchronizes. */
int cpt_tracer_read_image(cpt_tracer* t, float* rgba_host);
/* The same resolved image written to device memory (float4 per pixel, width x height
 * of the last raytrace, 16-B aligned) on the tracer's stream, without synchronizing:
 * for a caller that displays from device memory, as the reference's raytrace_kernel
 * writes its screen surface (cuda_path_tracer.cu:416-420) — e.g. followed by a
 * cudaMemcpy2DToArrayAsync into a graphics-interop array on cpt_tracer_stream(t). */
int cpt_tracer_resolve(cpt_tracer* t, float* rgba_dev);
/* Checkpoint / resume of the progressive image (the reference loses it on exit).
 * get: copies the accumulator of the last raytrace (cpt_accum_bytes(width, height,
 * accum_mode) bytes, the layout of the tracer's accum mode), the frame counter and
 * that accum mode (CPT_ACCUM_*) to host memory; synchronizes. set: restores them for a
 * width x height image, so that the next cpt_tracer_raytrace at that size continues
 * from frame `frame`; synchronizes. set refuses (CPT_ERR_INVALID_ARGUMENT) an
 * accum_mode other than the tracer's current one: the Kahan and FP64 layouts have the
 * same size, so the mode is checked rather than inferred. Resuming gives the same image
 * as an uninterrupted run when the scene, camera and settings (cpt_tracer_set_settings,
 * cpt_tracer_set_nee) are those of the saved run; apply the settings before set. A set
 * that fails leaves the tracer without an image (its next raytrace starts at frame 0). */
int cpt_tracer_get_progress(cpt_tracer* t, void* accum_host, size_t bytes, uint32_t* frame, uint32_t* accum_mode);
int cpt_tracer_set_progress(cpt_tracer* t, const void* accum_host, size_t bytes, uint32_t width, uint32_t height,
                            uint32_t frame, uint32_t accum_mode);
/* Rays traced since upload (primary, extension, shadow); synchronizes. */
int cpt_tracer_ray_counts(cpt_tracer* t, unsigned long long out[3]);
cudaStream_t cpt_tracer_stream(cpt_tracer* t);
const cpt_bvh* cpt_tracer_bvh(const cpt_tracer* t);

/* ---- synthetic scenes (host memory; the benchmark workloads) ---- */
/* Random triangles: centroids U[0,1]^3, edge lengths U(edge_min, edge_max) along
 * random unit vectors; plus a two-triangle emitter quad (light_size square at
 * light_y facing -y, emission light_emission) when light_size > 0.
 * albedo: grey vertex colour. Returns the triangle count written (n_random + 2). */
uint32_t cpt_scene_random(uint32_t n_random, uint32_t seed, float edge_min, float edge_max, float albedo,
                          float light_y, float light_size, float light_emission, cpt_triangle* tris,
                          cpt_triangle_info* infos);
/* Displaced sphere (lat-long grid nu x nv quads, radius 1 + amp * fBm) plus
 * n_hair thin random "hairball" triangles in a ball of radius hair_radius, plus
 * an emitter quad. Returns the triangle count (2*nu*nv + n_hair + 2). */
uint32_t cpt_scene_sphere_hairball(uint32_t nu, uint32_t nv, float amp, uint32_t n_hair, float hair_radius,
                                   uint32_t seed, float albedo, float light_y, float light_size,
                                   float light_emission, cpt_triangle* tris, cpt_triangle_info* infos);
/* Wavefront OBJ (+ MTL) ingest, as PathTracingApp::extractScene fills the scene
 * (PathTracingApp.cpp:31-124): world position = file position * scale + translate
 * (translate nullable), vertex colours or the material's Kd (default_grey without a
 * material), normals from the file or the triangle's geometric normal, Ke as
 * emission, Ns as specularity. With tris == NULL only counts: *n_out = triangles.
 * Returns CPT_ERR_SCRATCH_TOO_SMALL when capacity is below the count, and
 * CPT_ERR_INVALID_ARGUMENT for a missing file or a face whose position, uv or normal
 * index is 0 or outside the elements read so far. Host memory. */
int cpt_obj_load(const char* path, float scale, const float* translate, float default_grey, cpt_triangle* tris,
                 cpt_triangle_info* infos, uint32_t capacity, uint32_t* n_out);
/* Deforming-mesh workload (device memory): out = rest with every vertex moved
 * along its direction from the origin by amplitude * sin(omega * coord + phase). */
int cpt_scene_deform(const cpt_triangle* rest, cpt_triangle* out, uint32_t n, float amplitude, float omega,
                     float phase, cudaStream_t stream);
/* Enclosing box (min, max) of a host triangle soup, as the reference's caller builds it. */
void cpt_scene_bounds(const cpt_triangle* tris, uint32_t n, float out[6]);
/* Camera corner directions for eye/target/up, vertical fov (degrees), aspect,
 * near/far, with NDC jitter (jx, jy) — screenToRay (PathTracingApp.cpp:217-242).
 * Fills cam (dirs, eye, inv_view_proj; jitter fields left to the caller). */
void cpt_camera_look_at(const float eye[3], const float target[3], const float up[3], float fov_deg, float aspect,
                        float znear, float zfar, cpt_camera* cam);

/* ---- radiance cache (no reference counterpart: an extension measured by image
 * error against the FP64 estimator, with plain path tracing as fallback) ----
 * A 96 -> 4 x 64 (ReLU) -> 16 MLP (BF16 weights, FP32 accumulation) over the
 * encoded secondary vertex: 12-frequency sin/cos encoding of the position in the
 * scene box, real spherical harmonics bands 0-3 of the ray direction, normal,
 * albedo. It predicts the radiance that the rest of a path (vertices 2 and on)
 * brings to vertex 1, per unit throughput there; trained online with relative-L2
 * loss and Adam on full-depth training paths of the same renderer.
 * Samples (training and cpt_rc_infer) are 16 floats: position, target r,
 * direction, target g, normal, target b, albedo, 0. Weights (cpt_rc_get/set) are
 * FP32, per layer row-major [fan_in][fan_out], layers packed in order. */
typedef struct cpt_rc cpt_rc;
typedef struct cpt_rc_params {
    float learning_rate;     /* 1e-2 */
    float beta1, beta2;      /* 0.9, 0.99 */
    float epsilon;           /* 1e-15 */
    float ema_decay;         /* inference weights: 0 = the trained weights, else their moving average */
    uint32_t train_samples;  /* training paths per training frame, 65536 */
    uint32_t train_steps;    /* optimizer steps per training frame; the samples are split between them */
    uint32_t seed;           /* weight initialisation */
    uint32_t train_interval; /* cpt_rc_render trains on the frames whose first sample index / spp is a
                              * multiple of this (0 or 1: every frame); the other frames stop every path
                              * at vertex 1 and only read the cache */
} cpt_rc_params;
void cpt_rc_default_params(cpt_rc_params* p);
size_t cpt_rc_param_count(void);
int cpt_rc_create(cpt_rc** out, const cpt_rc_params* params /* nullable: defaults */, cudaStream_t stream);
void cpt_rc_destroy(cpt_rc* rc);
/* New random weights, optimizer state cleared. */
int cpt_rc_reset(cpt_rc* rc, uint32_t seed, cudaStream_t stream);
int cpt_rc_get_weights(cpt_rc* rc, float* host_out, cudaStream_t stream);
int cpt_rc_set_weights(cpt_rc* rc, const float* host_in, cudaStream_t stream);
/* Predictions for n device samples (16 floats each) -> out: n x (r, g, b, 0) on the device.
 * box: host (min xyz, max xyz) normalising positions. Synchronizes the stream. */
int cpt_rc_infer(cpt_rc* rc, const float* samples, uint32_t n, const float box[6], float* out, cudaStream_t stream);
/* `steps` optimizer steps over n device samples split into equal batches; *loss_out
 * (nullable) = mean relative L2 over the samples before their step. Synchronizes. */
int cpt_rc_train(cpt_rc* rc, const float* samples, uint32_t n, const float box[6], uint32_t steps, float* loss_out,
                 cudaStream_t stream);
/* One cached frame of the views (as cpt_render_views), training on its own paths:
 * about train_samples of the frame's paths, chosen by a hash of pixel and sample, are
 * traced to full depth — their estimate goes into the image and their radiance after
 * vertex 1 becomes a training target — and every other path is traced through vertex 1
 * and takes the cache's prediction for the rest; then train_steps optimizer steps over
 * the targets (used by the next frame). On frames that the train_interval skips, every
 * path takes the prediction and nothing is trained. bounces < 2 renders plain paths.
 * The position box is views[0].bvh's root box. */
size_t cpt_rc_render_scratch_bytes(const cpt_rc* rc, const cpt_view* views, uint32_t n_views,
                                   const cpt_render_params* params);
int cpt_rc_render(cpt_rc* rc, const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* scratch,
                  size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status, cudaStream_t stream);
/* The training half of cpt_rc_render alone (training paths + optimizer steps, no
 * image): warming a cache up, or following a scene change, without rendering. */
int cpt_rc_update(cpt_rc* rc, const cpt_view* views, uint32_t n_views, const cpt_render_params* params, void* scratch,
                  size_t scratch_bytes, unsigned long long* ray_counts, uint32_t* status, cudaStream_t stream);
/* Training samples collected by the last cpt_rc_render (device pointer, count). */
int cpt_rc_sample_count(cpt_rc* rc, uint32_t* out, cudaStream_t stream);
int cpt_rc_samples(cpt_rc* rc, const float** samples_dev);

/* ---- profiling: CUDA events around every kernel launch of the library ----
 * Between begin and end, each launch is bracketed by two events recorded on its
 * own stream. end() synchronizes those events and adds their elapsed times to
 * per-kernel totals, which get() reads by kernel name (e.g. "k_extend"). */
int cpt_profile_begin(void);
int cpt_profile_end(void);
int cpt_profile_get(const char* kernel, double* total_ms, unsigned long long* launches);
/* Milliseconds during which at least one launch of the kernel ran, between the last
 * begin and end (the union of the launches' event intervals; below the total when
 * launches on two streams overlap, e.g. two wave lanes). */
int cpt_profile_get_busy(const char* kernel, double* busy_ms);

/* ---- library info ---- */
const char* cpt_version(void);
/* Number of kernel launches the library has issued in this process. */
unsigned long long cpt_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
