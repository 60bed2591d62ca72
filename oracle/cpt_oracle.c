/* CPU oracle for the LBVH build and the path tracer. TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's hot path (compix/CUDA-Path-Tracer),
 * used by tests/ as the checker, by __graft_entry__.smoke() as the checker and by
 * bench.py's cpu_baseline leg when the reference itself was not compiled. The
 * product never links, loads or calls this file.
 *
 * Parity is pinned: tests/test_oracle_pin.py runs this restatement and the
 * reference's own builder and traversal (compiled from its sources into
 * oracle/_ref/libref.so by oracle/Makefile) on the same inputs and requires
 * identical bytes, and tests/golden/ holds fixtures produced by the reference.
 *
 * Arithmetic follows the reference's expressions operation by operation, with
 * glm 0.9.8's definitions spelled out (min(x,y) = x<y?x:y and max(x,y) = x>y?x:y,
 * func_common.inl:15-26; dot = (x*x' + y*y') + z*z', cross, normalize =
 * v * (1/sqrt(dot(v,v))), mix(x,y,a) = x + a*(y-x), func_geometric.inl:54-96,
 * func_exponential.inl:42-48, func_common.inl:143-151). The file is compiled with
 * -ffp-contract=off so every operation rounds on its own.
 *
 * Float to int conversion follows the GPU (cvt.rzi.s32.f32: NaN -> 0, saturating),
 * which is what the reference's morton_encoder does on its target; x86 host code
 * differs only for non-finite or out-of-range products (a zero-extent scene axis).
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include "cpt_rng.h"

/* ---- layouts (geometry.h:20-30, BBox.h:6-53, TriangleInfo.h:14-35, Lights.h) ---- */
typedef struct { float v0[3], v1[3], v2[3]; uint32_t info; } otri;          /* 40 B */
typedef struct { float mn[3], mx[3]; } obox;                                 /* 24 B */
typedef struct { float color[3], uv[2], normal[3], tangent[3], bitangent[3]; } overt; /* 56 B */
typedef struct { float emission[3]; float specularity; uint32_t albedo_idx, normal_idx; } omat;
typedef struct { overt v[3]; omat m; } oinfo;                                /* 192 B */
typedef struct { float color[3], dir[3], intensity; } olight;               /* 28 B */

#define INVALID_IDX 0xFFFFFFFFu
#define STACK_CAP 64 /* MAX_TRAVERSAL_STACK_SIZE, cuda_defs.h:21 */

int orc_sizeof_triangle(void) { return (int)sizeof(otri); }
int orc_sizeof_bbox(void) { return (int)sizeof(obox); }
int orc_sizeof_triangle_info(void) { return (int)sizeof(oinfo); }
int orc_sizeof_light(void) { return (int)sizeof(olight); }

static inline float gmin(float x, float y) { return x < y ? x : y; }
static inline float gmax(float x, float y) { return x > y ? x : y; }

/* ---- vec3 helpers: one IEEE operation each ---- */
typedef struct { float x, y, z; } v3;
static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 muls(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { float x = a.x * b.x, y = a.y * b.y, z = a.z * b.z; return x + y + z; }
static inline v3 cross(v3 a, v3 b)
{
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline v3 normalize(v3 v) { float s = 1.0f / sqrtf(dot(v, v)); return muls(v, s); }
/* math_util.h:19-23: v0*(1-u-v) + v1*u + v2*v */
static inline v3 bary(v3 a, v3 b, v3 c, float u, float v)
{
    float w = 1.0f - u - v;
    return add(add(muls(a, w), muls(b, u)), muls(c, v));
}
/* glm mix(x, y, a) = x + a*(y - x) */
static inline v3 mix3(v3 x, v3 y, float a) { return add(x, muls(sub(y, x), a)); }

/* ---- Morton codes (BVHBuilder.cu:12-32, math_util.h:10-13, morton.h:63-102) ---- */
static inline int32_t f2i_rz_sat(float x)
{
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}

static inline uint32_t quantize(float x, uint32_t n)
{
    int32_t q = f2i_rz_sat(x * (float)n);
    int32_t hi = (int32_t)(n - 1);
    q = q < hi ? q : hi;
    return (uint32_t)(q > 0 ? q : 0);
}

/* Bit interleave written as a loop: bit b of x/y/z goes to bit 3b/3b+1/3b+2. */
static inline uint64_t interleave3(uint32_t x, uint32_t y, uint32_t z, int order)
{
    uint64_t k = 0;
    for (int b = 0; b < order; ++b) {
        k |= (uint64_t)((x >> b) & 1u) << (3 * b);
        k |= (uint64_t)((y >> b) & 1u) << (3 * b + 1);
        k |= (uint64_t)((z >> b) & 1u) << (3 * b + 2);
    }
    return k;
}

static inline uint64_t morton_of(const otri* t, const float mn[3], const float inv[3], int order)
{
    uint32_t n = 1u << order, q[3];
    for (int a = 0; a < 3; ++a) {
        float c = (t->v0[a] + t->v1[a] + t->v2[a]) / 3.0f;
        q[a] = quantize((c - mn[a]) * inv[a], n);
    }
    return interleave3(q[0], q[1], q[2], order);
}

static void inv_scale(const float box[6], float inv[3])
{
    for (int a = 0; a < 3; ++a) inv[a] = 1.0f / (box[3 + a] - box[a]);
}

/* Morton keys of n triangles (bits 30 -> uint32 keys, 63 -> uint64 keys). */
void orc_morton(const otri* tris, uint32_t n, const float box[6], int bits, void* keys)
{
    float inv[3];
    inv_scale(box, inv);
    int order = bits == 30 ? 10 : 21;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) {
        uint64_t k = morton_of(&tris[i], box, inv, order);
        if (bits == 30) ((uint32_t*)keys)[i] = (uint32_t)k; else ((uint64_t*)keys)[i] = k;
    }
}

/* Enclosing box as the caller builds it (PathTracingApp.cpp:113): start from the
 * empty box (BBox.cpp:4-6) and unite every triangle's box in order. */
static inline void box_unite_pt(obox* b, const float* p)
{
    for (int a = 0; a < 3; ++a) { b->mn[a] = gmin(b->mn[a], p[a]); b->mx[a] = gmax(b->mx[a], p[a]); }
}
static inline void box_empty(obox* b)
{
    for (int a = 0; a < 3; ++a) { b->mn[a] = FLT_MAX; b->mx[a] = -FLT_MAX; }
}
static inline void box_unite(obox* b, const obox* c)
{
    for (int a = 0; a < 3; ++a) { b->mn[a] = gmin(b->mn[a], c->mn[a]); b->mx[a] = gmax(b->mx[a], c->mx[a]); }
}
static inline void tri_box(const otri* t, obox* b)
{
    box_empty(b);
    box_unite_pt(b, t->v0);
    box_unite_pt(b, t->v1);
    box_unite_pt(b, t->v2);
}

void orc_enclosing_box(const otri* tris, uint32_t n, float out[6])
{
    obox acc, tb;
    box_empty(&acc);
    for (uint32_t i = 0; i < n; ++i) { tri_box(&tris[i], &tb); box_unite(&acc, &tb); }
    memcpy(out, acc.mn, 3 * sizeof(float));
    memcpy(out + 3, acc.mx, 3 * sizeof(float));
}

/* ---- stable key sort (thrust::sort_by_key, BVHBuilder.cu:234) ---- */
typedef struct { uint64_t key; uint32_t idx; } kv;
static int kv_cmp(const void* a, const void* b)
{
    const kv* x = (const kv*)a; const kv* y = (const kv*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->idx < y->idx ? -1 : (x->idx > y->idx);
}

/* ---- Karras radix tree (BVHBuilder.cu:107-201) ---- */
static inline int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

static inline int delta(const uint64_t* k, uint32_t n, int i, int j, int total_bits)
{
    if (j < 0 || (uint32_t)j >= n) return -1;
    if (k[i] == k[j]) return clz32((uint32_t)(i ^ j)) + total_bits;
    return total_bits == 32 ? clz32((uint32_t)(k[i] ^ k[j])) : clz64(k[i] ^ k[j]);
}

static void radix_tree(const uint64_t* k, uint32_t n, int total_bits, uint32_t* children,
                       uint32_t* parents_leaf, uint32_t* parents_internal)
{
    parents_internal[0] = INVALID_IDX; /* BVHBuilder.cu:224 */
#pragma omp parallel for schedule(static)
    for (long ii = 0; ii < (long)n - 1; ++ii) {
        int i = (int)ii;
        int dd = delta(k, n, i, i + 1, total_bits) - delta(k, n, i, i - 1, total_bits);
        int d = (dd > 0) - (dd < 0);
        int dmin = delta(k, n, i, i - d, total_bits);
        int lmax = 2;
        while (delta(k, n, i, i + lmax * d, total_bits) > dmin) lmax *= 2;
        int l = 0;
        while (lmax > 1) {
            lmax /= 2;
            if (delta(k, n, i, i + (l + lmax) * d, total_bits) > dmin) l += lmax;
        }
        int j = i + l * d;
        int dnode = delta(k, n, i, j, total_bits);
        int s = 0;
        while (l > 1) {
            l = (l + 1) / 2;
            if (delta(k, n, i, i + (s + l) * d, total_bits) > dnode) s += l;
        }
        s = i + s * d + (d < 0 ? d : 0);
        uint32_t type = 0;
        int lo = i < j ? i : j, hi = i > j ? i : j;
        if (lo != s) { type |= 1u; parents_internal[s] = (uint32_t)i; }
        else parents_leaf[s] = (uint32_t)i;
        if (hi != s + 1) { type |= 2u; parents_internal[s + 1] = (uint32_t)i; }
        else parents_leaf[s + 1] = (uint32_t)i;
        children[i] = ((uint32_t)s << 2) | type;
    }
}

/* ---- bottom-up AABB refit (BVHBuilder.cu:39-98), leaves visited in index order;
 *      every internal box is left.unite(right) whatever the visiting order ---- */
static void refit(const otri* sorted, uint32_t n, const uint32_t* children, const uint32_t* parents_leaf,
                  const uint32_t* parents_internal, obox* boxes)
{
    int* counters = (int*)calloc(n, sizeof(int));
    for (uint32_t leaf = 0; leaf < n; ++leaf) {
        uint32_t cur = parents_leaf[leaf];
        while (cur != INVALID_IDX) {
            if (counters[cur]++ == 0) break;
            uint32_t node = children[cur];
            uint32_t li = node >> 2, ri = li + 1;
            obox lb, rb;
            if ((node & 1u) == 0) tri_box(&sorted[li], &lb); else lb = boxes[li];
            if ((node & 2u) == 0) tri_box(&sorted[ri], &rb); else rb = boxes[ri];
            box_unite(&lb, &rb);
            boxes[cur] = lb;
            cur = parents_internal[cur];
        }
    }
    free(counters);
}

/* Full LBVH build: Morton codes, stable sort (triangles permuted), topology,
 * refit. Outputs are the reference's arrays. Returns 0, or -1 for n < 2 or bad bits. */
int orc_build(const otri* tris_in, uint32_t n, const float box[6], int bits, otri* tris_out,
              void* keys_out, uint32_t* children, uint32_t* parents_leaf, uint32_t* parents_internal,
              obox* node_boxes)
{
    if (n < 2 || (bits != 30 && bits != 63)) return -1;
    float inv[3];
    inv_scale(box, inv);
    int order = bits == 30 ? 10 : 21;
    kv* a = (kv*)malloc(sizeof(kv) * n);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n; ++i) { a[i].key = morton_of(&tris_in[i], box, inv, order); a[i].idx = (uint32_t)i; }
    qsort(a, n, sizeof(kv), kv_cmp);
    uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * n);
    for (uint32_t i = 0; i < n; ++i) {
        tris_out[i] = tris_in[a[i].idx];
        k[i] = a[i].key;
        if (bits == 30) ((uint32_t*)keys_out)[i] = (uint32_t)a[i].key; else ((uint64_t*)keys_out)[i] = a[i].key;
    }
    free(a);
    radix_tree(k, n, bits == 30 ? 32 : 64, children, parents_leaf, parents_internal);
    free(k);
    refit(tris_out, n, children, parents_leaf, parents_internal, node_boxes);
    return 0;
}

/* ---- traversal (trace.h:73-180, intersection.h:28-59 and 106-117) ---- */
typedef struct {
    const otri* tris;
    const uint32_t* children;
    const obox* boxes;
    uint32_t n;
} obvh;

static inline int mt_hit(v3 o, v3 d, const otri* tri, float* u_out, float* v_out, float* t_out)
{
    v3 p0 = ld3(tri->v0), p1 = ld3(tri->v1), p2 = ld3(tri->v2);
    v3 e1 = sub(p1, p0), e2 = sub(p2, p0);
    v3 q = cross(d, e2);
    float det = dot(e1, q);
    if (det > -FLT_EPSILON && det < FLT_EPSILON) return 0;
    float inv = 1.f / det;
    v3 s = sub(o, p0);
    float u = inv * dot(s, q);
    *u_out = u;
    if (u < 0.f) return 0;
    v3 r = cross(s, e1);
    float v = inv * dot(d, r);
    *v_out = v;
    if (v < 0.f || (u + v) > 1.f) return 0;
    float t = inv * dot(e2, r);
    *t_out = t;
    return t >= 0.0f;
}

static inline int slab_hit(v3 o, v3 dinv, const obox* b, float* t_out)
{
    v3 tmn = mul(sub(ld3(b->mn), o), dinv);
    v3 tmx = mul(sub(ld3(b->mx), o), dinv);
    v3 t1 = mk(gmin(tmn.x, tmx.x), gmin(tmn.y, tmx.y), gmin(tmn.z, tmx.z));
    v3 t2 = mk(gmax(tmn.x, tmx.x), gmax(tmn.y, tmx.y), gmax(tmn.z, tmx.z));
    float tn = gmax(gmax(t1.x, t1.y), t1.z);
    float tf = gmin(gmin(t2.x, t2.y), t2.z);
    *t_out = tn;
    return tn <= tf && tf > 0.0f;
}

typedef struct { uint64_t nodes, box_tests, tri_tests, overflow; uint32_t max_depth; } ostats;

/* Child test of computeNodeIntersection (trace.h:60-71): FLT_MAX on a miss. */
static inline float child_hit(const obvh* b, v3 o, v3 d, v3 dinv, uint32_t idx, int internal, float* u,
                              float* v, ostats* st)
{
    float t;
    if (internal) {
        st->box_tests++;
        if (slab_hit(o, dinv, &b->boxes[idx], &t)) return t;
    } else {
        st->tri_tests++;
        if (mt_hit(o, d, &b->tris[idx], u, v, &t)) return t;
    }
    return FLT_MAX;
}

/* Closest hit (any_hit = 0) or first hit (any_hit = 1; same visiting order, stops
 * at the first recorded triangle, so its hit/miss equals the closest-hit's). */
static float trace_ray_lim(const obvh* b, v3 o, v3 d, int any_hit, float tmax, uint32_t* idx_out, float* u_out,
                           float* v_out, ostats* st)
{
    v3 dinv = mk(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    uint32_t stack[STACK_CAP];
    int top = 0;
    stack[top++] = 0u; /* Node::makeInternal(0): the root */
    float best = tmax; /* FLT_MAX: unbounded; otherwise a hit must lie nearer than tmax */
    uint32_t best_idx = INVALID_IDX;
    float bu = 0.f, bv = 0.f;
    while (top > 0) {
        uint32_t cur = stack[--top];
        for (;;) {
            uint32_t node = b->children[cur];
            st->nodes++;
            uint32_t ci[2] = {node >> 2, (node >> 2) + 1};
            int cint[2] = {(int)(node & 1u), (int)((node >> 1) & 1u)};
            float h[2], us[2] = {0.f, 0.f}, vs[2] = {0.f, 0.f};
            h[0] = child_hit(b, o, d, dinv, ci[0], cint[0], &us[0], &vs[0], st);
            h[1] = child_hit(b, o, d, dinv, ci[1], cint[1], &us[1], &vs[1], st);
            if (h[0] >= best && h[1] >= best) break;
            int c = 0, f = 1;
            if (h[1] < h[0]) { c = 1; f = 0; }
            if (cint[c]) {
                uint32_t next = ci[c];
                if (h[f] < best) {
                    if (cint[f]) {
                        if (top == STACK_CAP) st->overflow++;
                        else stack[top++] = ci[f];
                        if ((uint32_t)top > st->max_depth) st->max_depth = (uint32_t)top;
                    } else {
                        best = h[f]; bu = us[f]; bv = vs[f]; best_idx = ci[f];
                        if (any_hit) goto done;
                    }
                }
                cur = next;
            } else {
                best = h[c]; bu = us[c]; bv = vs[c]; best_idx = ci[c];
                if (any_hit) goto done;
                break;
            }
        }
    }
done:
    *idx_out = best_idx;
    *u_out = bu;
    *v_out = bv;
    return best;
}

static float trace_ray(const obvh* b, v3 o, v3 d, int any_hit, uint32_t* idx_out, float* u_out, float* v_out,
                       ostats* st)
{
    return trace_ray_lim(b, o, d, any_hit, FLT_MAX, idx_out, u_out, v_out, st);
}

/* rays: m x 6 floats (origin, direction). Outputs per ray: t (FLT_MAX on miss),
 * sorted-leaf triangle index (0xFFFFFFFF on miss), uv. stats (nullable): 5 u64 per
 * ray — internal nodes fetched, box tests, triangle tests, stack overflows, max depth. */
void orc_trace(const otri* sorted, const uint32_t* children, const obox* boxes, uint32_t n, const float* rays,
               uint32_t m, int any_hit, float* t_out, uint32_t* idx_out, float* uv_out, uint64_t* stats)
{
    obvh b = {sorted, children, boxes, n};
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)m; ++i) {
        ostats st = {0, 0, 0, 0, 0};
        float u, v;
        uint32_t idx;
        float t = trace_ray(&b, ld3(rays + 6 * i), ld3(rays + 6 * i + 3), any_hit, &idx, &u, &v, &st);
        t_out[i] = t;
        idx_out[i] = idx;
        if (uv_out) { uv_out[2 * i] = u; uv_out[2 * i + 1] = v; }
        if (stats) {
            uint64_t* s = stats + 5 * i;
            s[0] = st.nodes; s[1] = st.box_tests; s[2] = st.tri_tests; s[3] = st.overflow; s[4] = st.max_depth;
        }
    }
}

/* ---- path tracer (cuda_path_tracer.cu:36-50, 115-220, 245-333, 376-421) ---- */
typedef struct {
    obvh bvh;
    const oinfo* infos;
    const olight* lights;
    uint32_t light_count;
    uint32_t bounces;
    float intensity;
    int stratified;
    uint32_t k0, k1;
    uint32_t camera;  /* counter word 3 of the bounce stream */
} oscene;

/* ---- textures: Scene::upload's sampler (Scene.cu:57-81) read by extractInfo /
 * unpackNormal (cuda_path_tracer.cu:85-138) ---- */
typedef struct { const uint8_t* rgba; uint32_t width, height; } otex;
static const otex* g_textures;
static uint32_t g_texture_count;

/* The texture table later renders read (NULL clears it). */
void orc_set_textures(const otex* textures, uint32_t count)
{
    g_textures = textures;
    g_texture_count = textures ? count : 0;
}

/* tex2D<float4> with normalized coordinates, wrap addressing, bilinear filtering and
 * normalized-float reads of RGBA8 texels, as the CUDA C Programming Guide states
 * texture fetching ("Texture Fetching", linear filtering): wrap takes frac(u); the
 * texel-space position is x = frac(u) * W - 0.5, i = floor(x), and the weight
 * a = frac(x) is held in 9-bit fixed point with 8 fraction bits (rounded to
 * nearest here; the hardware's rounding of that step is not documented, which the
 * parity tests' tolerance covers). Texel values are byte / 255. */
static void tex_sample(const otex* t, double u, double v, double out[4])
{
    double x = (u - floor(u)) * (double)t->width - 0.5, y = (v - floor(v)) * (double)t->height - 0.5;
    double fx = floor(x), fy = floor(y);
    double a = nearbyint((x - fx) * 256.0) / 256.0, b = nearbyint((y - fy) * 256.0) / 256.0;
    long W = (long)t->width, H = (long)t->height;
    long i0 = (((long)fx % W) + W) % W, j0 = (((long)fy % H) + H) % H;
    long i1 = (i0 + 1) % W, j1 = (j0 + 1) % H;
    const uint8_t* p00 = t->rgba + 4 * (j0 * W + i0);
    const uint8_t* p10 = t->rgba + 4 * (j0 * W + i1);
    const uint8_t* p01 = t->rgba + 4 * (j1 * W + i0);
    const uint8_t* p11 = t->rgba + 4 * (j1 * W + i1);
    for (int c = 0; c < 4; ++c)
        out[c] = ((1.0 - a) * (1.0 - b) * p00[c] + a * (1.0 - b) * p10[c] + (1.0 - a) * b * p01[c] + a * b * p11[c]) /
                 255.0;
}

/* tex_sample for n coordinate pairs (tests of the sampler alone). */
void orc_tex_sample(const otex* t, const float* uv, uint32_t n, float* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        double s[4];
        tex_sample(t, uv[2 * i], uv[2 * i + 1], s);
        for (int c = 0; c < 4; ++c) out[4 * i + c] = (float)s[c];
    }
}

/* extractInfo + unpackNormal (cuda_path_tracer.cu:85-138): albedo from the albedo
 * texture at the interpolated uv, else the normalised interpolated colour; normal
 * from the normal map in the interpolated tangent frame, else the normalised
 * interpolated normal. An index past the texture table counts as absent. */
static void surface(const oinfo* in, float u, float v, v3* albedo, v3* normal)
{
    *normal = normalize(bary(ld3(in->v[0].normal), ld3(in->v[1].normal), ld3(in->v[2].normal), u, v));
    uint32_t ai = in->m.albedo_idx, ni = in->m.normal_idx;
    int ta = ai < g_texture_count, tn = ni < g_texture_count;
    if (!ta) *albedo = normalize(bary(ld3(in->v[0].color), ld3(in->v[1].color), ld3(in->v[2].color), u, v));
    if (!ta && !tn) return;
    float w = (1.0f - u) - v;
    float tu = (in->v[0].uv[0] * w + in->v[1].uv[0] * u) + in->v[2].uv[0] * v;
    float tv = (in->v[0].uv[1] * w + in->v[1].uv[1] * u) + in->v[2].uv[1] * v;
    double s[4];
    if (ta) {
        tex_sample(&g_textures[ai], tu, tv, s);
        *albedo = mk((float)s[0], (float)s[1], (float)s[2]);
    }
    if (tn) {
        tex_sample(&g_textures[ni], tu, tv, s);
        float nx = 2.0f * (float)s[0] - 1.0f, ny = 2.0f * (float)s[1] - 1.0f, nz = 2.0f * (float)s[2] - 1.0f;
        v3 tg = normalize(bary(ld3(in->v[0].tangent), ld3(in->v[1].tangent), ld3(in->v[2].tangent), u, v));
        v3 bt = normalize(bary(ld3(in->v[0].bitangent), ld3(in->v[1].bitangent), ld3(in->v[2].bitangent), u, v));
        *normal = normalize(add(add(muls(tg, nx), muls(bt, ny)), muls(*normal, nz)));
    }
}

typedef struct { uint64_t primary, extension, shadow; } ocount;

static inline float emission_sum(const omat* m) { return m->emission[0] + m->emission[1] + m->emission[2]; }

/* computeL (LightAlgorithms.h:12-20): full-trace visibility toward -dir. */
static inline v3 light_l(const oscene* sc, v3 p, const olight* l, ocount* cnt)
{
    v3 dir = ld3(l->dir);
    v3 o = sub(p, muls(dir, 1e-3f));
    uint32_t idx; float u, v;
    ostats st = {0, 0, 0, 0, 0};
    float dist = trace_ray(&sc->bvh, o, neg(dir), 1, &idx, &u, &v, &st);
    cnt->shadow++;
    if (dist < FLT_MAX) return mk(0.f, 0.f, 0.f);
    return muls(ld3(l->color), l->intensity);
}

/* blinnPhongBRDF (cuda_path_tracer.cu:36-50) */
static inline v3 blinn_phong(v3 Id, v3 kd, v3 Is, v3 ks, v3 n, v3 lv, v3 h, float shininess)
{
    float df = gmax(dot(n, lv), 0.0f);
    v3 diffuse = muls(mul(Id, kd), df);
    float sf = powf(gmax(dot(n, h), 0.0f), shininess);
    v3 spec = mk(0.f, 0.f, 0.f);
    if (shininess > 0.0 && df > 0.0f) spec = muls(mul(Is, ks), sf);
    return add(diffuse, spec);
}

/* toHemisphere (math_util.h:56-67) */
static inline v3 to_hemisphere(v3 vec, v3 n)
{
    v3 x;
    if (fabsf(n.x) < FLT_EPSILON) x = cross(n, mk(1.0f, 0.0f, 0.0f));
    else x = cross(n, mk(0.0f, 1.0f, 0.0f));
    x = normalize(x);
    v3 y = normalize(cross(n, x));
    return add(add(muls(x, vec.x), muls(y, vec.y)), muls(n, vec.z));
}

static inline const oinfo* info_of(const oscene* sc, uint32_t sorted_idx)
{
    return &sc->infos[sc->bvh.tris[sorted_idx].info];
}

/* ---- next-event estimation (an extension of the renderer, no reference counterpart) ----
 * Emitter table, restated from the product's layout: a 16-B header (count, total
 * area, emitters found, overflow flag) and 48 B per emitter, (v0, cdf)
 * (v1 - v0, area) (v2 - v0, sorted triangle index), the emissive triangles
 * (emission r + g + b > 1e-7) in sorted order; area = 0.5 |e1 x e2|; cdf summed
 * in segments of 256 emitters (partial sums in each segment, then the segment
 * totals in order), cdf_j = (segment offset + partial sum) / total.
 * Returns the number of emitters found; the table holds them when <= cap. */
#define NEE_SEG 256u
uint32_t orc_emitters(const otri* sorted, uint32_t n, const oinfo* infos, uint32_t info_count, uint32_t cap,
                      float* table)
{
    uint32_t found = 0;
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t ii = sorted[i].info;
        if (ii < info_count && emission_sum(&infos[ii].m) > 1e-7f) ++found;
    }
    uint32_t count = found <= cap ? found : 0u, overflow = found <= cap ? 0u : 1u;
    float* rec = table + 4;
    uint32_t j = 0;
    for (uint32_t i = 0; i < n && count; ++i) {
        uint32_t ii = sorted[i].info;
        if (!(ii < info_count && emission_sum(&infos[ii].m) > 1e-7f)) continue;
        v3 v0 = ld3(sorted[i].v0), e1 = sub(ld3(sorted[i].v1), v0), e2 = sub(ld3(sorted[i].v2), v0);
        v3 c = cross(e1, e2);
        float* r = rec + 12 * (size_t)j++;
        r[0] = v0.x; r[1] = v0.y; r[2] = v0.z; r[3] = 0.f;
        r[4] = e1.x; r[5] = e1.y; r[6] = e1.z; r[7] = 0.5f * sqrtf(dot(c, c));
        r[8] = e2.x; r[9] = e2.y; r[10] = e2.z; memcpy(&r[11], &i, 4);
    }
    float total = 0.f;
    uint32_t segs = (count + NEE_SEG - 1) / NEE_SEG;
    for (uint32_t sgi = 0; sgi < segs; ++sgi) {
        float seg = 0.f;
        for (uint32_t k = sgi * NEE_SEG; k < count && k < (sgi + 1) * NEE_SEG; ++k) seg += rec[12 * (size_t)k + 7];
        total += seg;
    }
    float off = 0.f;
    for (uint32_t sgi = 0; sgi < segs; ++sgi) {
        float sum = 0.f;
        for (uint32_t k = sgi * NEE_SEG; k < count && k < (sgi + 1) * NEE_SEG; ++k) {
            sum += rec[12 * (size_t)k + 7];
            rec[12 * (size_t)k + 3] = total > 0.f ? (off + sum) / total : 0.f;
        }
        off += sum;
    }
    memcpy(&table[0], &count, 4);
    table[1] = total;
    memcpy(&table[2], &found, 4);
    memcpy(&table[3], &overflow, 4);
    return found;
}

/* The emitter table later renders estimate direct light with (NULL: the
 * reference's estimator). */
static const float* g_nee;
void orc_set_nee(const float* table) { g_nee = table; }

/* One emitter draw at a vertex that bounces (origin no of its bounce, shading
 * normal n, path weight absorbed): a point y drawn with density 1 / A, the
 * estimate intensity * absorbed * e * max(-w . n_e, 0) * (n . w / pi) *
 * |n_g . w| / r^2 * A of the emission the bounce would pick up, and the shadow
 * ray toward y (direction w, far limit 0.9999 r). Returns 0 when the estimate is 0. */
static int nee_sample(const oscene* sc, v3 no, v3 n, v3 absorbed, uint32_t pixel, uint32_t frame, uint32_t depth,
                      v3* c_out, v3* w_out, float* tmax)
{
    uint32_t count;
    memcpy(&count, g_nee, 4);
    float total = g_nee[1];
    if (count == 0 || !(total > 0.0f)) return 0;
    float up, s1, s2;
    cpt_rng_nee_uniforms(sc->k0, sc->k1, pixel, frame, depth, sc->camera, &up, &s1, &s2);
    const float* rec = g_nee + 4;
    uint32_t lo = 0, hi = count - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (up < rec[12 * (size_t)mid + 3]) hi = mid;
        else lo = mid + 1;
    }
    const float* r = rec + 12 * (size_t)lo;
    v3 v0 = ld3(r), e1 = ld3(r + 4), e2 = ld3(r + 8);
    uint32_t tri;
    memcpy(&tri, &r[11], 4);
    float sq = sqrtf(s1);
    float bu = sq * (1.0f - s2), bw = sq * s2;
    v3 y = add(add(v0, muls(e1, bu)), muls(e2, bw));
    v3 dv = sub(y, no);
    float r2 = dot(dv, dv);
    if (!(r2 > 0.0f)) return 0;
    float dist = sqrtf(r2);
    v3 w = muls(dv, 1.0f / dist);
    float cos_x = dot(n, w);
    if (!(cos_x > 0.0f)) return 0;
    const oinfo* in = info_of(sc, tri);
    v3 ae, ne;
    surface(in, bu, bw, &ae, &ne);
    float cos_e = gmax(dot(neg(w), ne), 0.0f);
    if (!(cos_e > 0.0f)) return 0;
    float cos_g = fabsf(dot(normalize(cross(e1, e2)), w));
    float g = (((cos_x * cos_e) * cos_g) * total) / (r2 * 3.14159265358979f);
    *c_out = muls(mul(absorbed, ld3(in->m.emission)), g * sc->intensity);
    *w_out = w;
    *tmax = dist * 0.9999f;
    return 1;
}

/* One path (blinnPhongShadingPathTrace, cuda_path_tracer.cu:245-333). */
static v3 path_radiance(const oscene* sc, v3 o, v3 d, uint32_t pixel, uint32_t frame, ocount* cnt)
{
    uint32_t idx; float u, v;
    ostats st = {0, 0, 0, 0, 0};
    float t = trace_ray(&sc->bvh, o, d, 0, &idx, &u, &v, &st);
    cnt->primary++;
    if (idx == INVALID_IDX) return mk(0.f, 0.f, 0.f);
    const oinfo* in = info_of(sc, idx);
    v3 hit = add(muls(d, t), o);
    v3 albedo, normal;
    surface(in, u, v, &albedo, &normal);
    v3 acc;
    if (emission_sum(&in->m) > 1e-7f) {
        albedo = mk(1.f, 1.f, 1.f);
        acc = ld3(in->m.emission);
    } else {
        v3 L = mk(0.f, 0.f, 0.f), color = mk(0.f, 0.f, 0.f);
        for (uint32_t i = 0; i < sc->light_count; ++i) {
            const olight* l = &sc->lights[i];
            L = add(L, light_l(sc, hit, l, cnt));
            v3 view = neg(d);
            v3 half = muls(sub(view, ld3(l->dir)), 0.5f);
            color = add(color, blinn_phong(L, albedo, L, mk(0.5f, 0.5f, 0.5f), normal, neg(ld3(l->dir)), half,
                                           in->m.specularity));
        }
        acc = color;
    }
    v3 absorbed = albedo;
    for (uint32_t i = 0; i < sc->bounces; ++i) {
        v3 ro = add(hit, muls(normal, 1e-5f));
        if (g_nee) {
            v3 c, w;
            float tmax;
            if (nee_sample(sc, ro, normal, absorbed, pixel, frame, i, &c, &w, &tmax)) {
                uint32_t si;
                float su, sv;
                trace_ray_lim(&sc->bvh, ro, w, 1, tmax, &si, &su, &sv, &st);
                cnt->shadow++;
                if (si == INVALID_IDX) acc = add(acc, c);
            }
        }
        float u0, u1;
        cpt_rng_bounce_uniforms(sc->k0, sc->k1, pixel, frame, i, sc->camera, &u0, &u1);
        float rx = u0, ry = u1;
        if (sc->stratified && i == 0) {
            uint32_t pos = frame % 64u;
            rx = ((float)(int)(pos % 8u) + u0) / 8.0f;
            ry = ((float)(int)(pos / 8u) + u1) / 8.0f;
        }
        float sn, cs;
        cpt_sincos_turns(ry, &sn, &cs);
        float r = sqrtf(rx);
        v3 rd = mk(r * cs, r * sn, sqrtf(1.0f - rx));
        rd = to_hemisphere(rd, normal);
        t = trace_ray(&sc->bvh, ro, rd, 0, &idx, &u, &v, &st);
        cnt->extension++;
        if (idx == INVALID_IDX) break;
        hit = add(muls(rd, t), ro);
        in = info_of(sc, idx);
        surface(in, u, v, &albedo, &normal);
        v3 L = mk(0.f, 0.f, 0.f);
        if (emission_sum(&in->m) > 1e-7f) {
            if (!g_nee) L = muls(ld3(in->m.emission), gmax(dot(neg(rd), normal), 0.0f));
            albedo = mk(1.f, 1.f, 1.f);
        } else {
            for (uint32_t l = 0; l < sc->light_count; ++l) {
                const olight* li = &sc->lights[l];
                v3 c = light_l(sc, hit, li, cnt);
                L = add(L, muls(c, gmax(dot(neg(ld3(li->dir)), normal), 0.0f)));
            }
        }
        absorbed = mul(absorbed, albedo);
        acc = add(acc, muls(mul(absorbed, L), sc->intensity));
    }
    return acc;
}

/* Camera: eye + four corner directions (00, 10, 11, 01) as
 * CUDAPathTracer::setPrimaryRays, or — when jitter is on — corner directions
 * re-derived per sample from the inverse view-projection with an NDC offset
 * drawn from the jitter stream (the per-frame jitter of screenToRay,
 * PathTracingApp.cpp:217-242, with inverse(T*VP) = inverse(VP)*inverse(T)). */
typedef struct {
    float eye[3];
    float dirs[4][3];
    float inv_view_proj[16]; /* column-major, as glm */
    float jitter_x, jitter_y; /* NDC half-range, 2/W and 2/H in the reference */
    uint32_t jitter;
} ocam;

static inline void mat_vec(const float* m, const float v[4], float r[4])
{
    for (int row = 0; row < 4; ++row) {
        float a = m[0 * 4 + row] * v[0];
        float b = m[1 * 4 + row] * v[1];
        float c = m[2 * 4 + row] * v[2];
        float d = m[3 * 4 + row] * v[3];
        r[row] = a + b + c + d;
    }
}

void orc_corner_dirs(const ocam* cam, uint32_t k0, uint32_t k1, uint32_t sample, float out[4][3])
{
    if (!cam->jitter) { memcpy(out, cam->dirs, sizeof(float) * 12); return; }
    float u0, u1;
    cpt_rng_jitter_uniforms(k0, k1, sample, &u0, &u1);
    float jx = (2.0f * u0 - 1.0f) * cam->jitter_x;
    float jy = (2.0f * u1 - 1.0f) * cam->jitter_y;
    static const float cx[4] = {-1.f, 1.f, 1.f, -1.f}, cy[4] = {-1.f, -1.f, 1.f, 1.f};
    for (int c = 0; c < 4; ++c) {
        float s[4] = {cx[c] - jx, cy[c] - jy, -1.0f, 1.0f}, e[4] = {cx[c] - jx, cy[c] - jy, 1.0f, 1.0f};
        float ws[4], we[4];
        mat_vec(cam->inv_view_proj, s, ws);
        mat_vec(cam->inv_view_proj, e, we);
        v3 ps = mk(ws[0] / ws[3], ws[1] / ws[3], ws[2] / ws[3]);
        v3 pe = mk(we[0] / we[3], we[1] / we[3], we[2] / we[3]);
        v3 dd = normalize(sub(pe, ps));
        out[c][0] = dd.x; out[c][1] = dd.y; out[c][2] = dd.z;
    }
}

/* Renders samples frame0 .. frame0+spp-1 of rows [row0, row1) and writes each
 * sample's radiance (3 floats) to radiance[(s * rows + (y - row0)) * width + x].
 * camera: the camera index of a multi-camera render (random-stream word 3).
 * Pixels are indexed p = y*width + x for the random streams. counts (nullable):
 * primary, extension, shadow rays. */
void orc_render(const otri* sorted, const uint32_t* children, const obox* boxes, uint32_t n, const oinfo* infos,
                const olight* lights, uint32_t light_count, uint32_t width, uint32_t height, uint32_t row0,
                uint32_t row1, uint32_t spp, uint32_t frame0, uint32_t bounces, float intensity, int stratified,
                uint32_t k0, uint32_t k1, const ocam* cam, uint32_t camera, float* radiance, uint64_t* counts)
{
    oscene sc = {{sorted, children, boxes, n}, infos, lights, light_count, bounces, intensity, stratified, k0, k1,
                 camera};
    uint32_t rows = row1 - row0;
    uint64_t tp = 0, te = 0, ts = 0;
    (void)height;
    for (uint32_t s = 0; s < spp; ++s) {
        float dirs[4][3];
        orc_corner_dirs(cam, k0, k1, frame0 + s, dirs);
        v3 d00 = ld3(dirs[0]), d10 = ld3(dirs[1]), d11 = ld3(dirs[2]), d01 = ld3(dirs[3]);
        v3 eye = ld3(cam->eye);
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tp, te, ts)
        for (long q = 0; q < (long)rows * width; ++q) {
            uint32_t x = (uint32_t)(q % width), y = row0 + (uint32_t)(q / width);
            float tx = (float)x / (float)width, ty = (float)y / (float)height;
            v3 dir = mix3(mix3(d00, d10, tx), mix3(d01, d11, tx), ty);
            ocount cnt = {0, 0, 0};
            v3 r = path_radiance(&sc, eye, dir, y * width + x, frame0 + s, &cnt);
            float* o = radiance + ((size_t)s * rows * width + (size_t)q) * 3;
            o[0] = r.x; o[1] = r.y; o[2] = r.z;
            tp += cnt.primary; te += cnt.extension; ts += cnt.shadow;
        }
    }
    if (counts) { counts[0] = tp; counts[1] = te; counts[2] = ts; }
}

/* ---- FP64 twin of the estimator (for RMSE); same sampling, double arithmetic ---- */
typedef struct { double x, y, z; } d3;
static inline d3 dmk(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static inline d3 dld(const float* p) { return dmk(p[0], p[1], p[2]); }
static inline d3 dadd(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline d3 dsub(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline d3 dmul(d3 a, d3 b) { return dmk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline d3 dmuls(d3 a, double s) { return dmk(a.x * s, a.y * s, a.z * s); }
static inline double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline d3 dcross(d3 a, d3 b) { return dmk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y); }
static inline d3 dnorm(d3 v) { return dmuls(v, 1.0 / sqrt(ddot(v, v))); }
static inline d3 dbary(d3 a, d3 b, d3 c, double u, double v) { return dadd(dadd(dmuls(a, 1.0 - u - v), dmuls(b, u)), dmuls(c, v)); }

static int mt_hit_d(d3 o, d3 d, const otri* tri, double* u_out, double* v_out, double* t_out)
{
    d3 p0 = dld(tri->v0), e1 = dsub(dld(tri->v1), p0), e2 = dsub(dld(tri->v2), p0);
    d3 q = dcross(d, e2);
    double det = ddot(e1, q);
    if (det > -FLT_EPSILON && det < FLT_EPSILON) return 0;
    double inv = 1.0 / det;
    d3 s = dsub(o, p0);
    double u = inv * ddot(s, q);
    if (u < 0.0) return 0;
    d3 r = dcross(s, e1);
    double v = inv * ddot(d, r);
    if (v < 0.0 || u + v > 1.0) return 0;
    double t = inv * ddot(e2, r);
    *u_out = u; *v_out = v; *t_out = t;
    return t >= 0.0;
}

static int slab_hit_d(d3 o, d3 dinv, const obox* b, double* t_out)
{
    double tn = -INFINITY, tf = INFINITY;
    double oo[3] = {o.x, o.y, o.z}, di[3] = {dinv.x, dinv.y, dinv.z};
    for (int a = 0; a < 3; ++a) {
        double t0 = (b->mn[a] - oo[a]) * di[a], t1 = (b->mx[a] - oo[a]) * di[a];
        double lo = t0 < t1 ? t0 : t1, hi = t0 > t1 ? t0 : t1;
        if (lo != lo) lo = -INFINITY;
        if (hi != hi) hi = INFINITY;
        tn = lo > tn ? lo : tn;
        tf = hi < tf ? hi : tf;
    }
    *t_out = tn;
    return tn <= tf && tf > 0.0;
}

/* Exhaustive-order-free closest hit in double: same tree, best-first pruning. */
static double trace_d(const obvh* b, d3 o, d3 d, int any_hit, uint32_t* idx_out, double* u_out, double* v_out)
{
    d3 dinv = dmk(1.0 / d.x, 1.0 / d.y, 1.0 / d.z);
    uint32_t stack[256];
    int top = 0;
    stack[top++] = 0u;
    double best = INFINITY;
    uint32_t bi = INVALID_IDX;
    double bu = 0, bv = 0;
    while (top > 0) {
        uint32_t cur = stack[--top];
        uint32_t node = b->children[cur];
        for (int c = 0; c < 2; ++c) {
            uint32_t ci = (node >> 2) + (uint32_t)c;
            int internal = c == 0 ? (int)(node & 1u) : (int)((node >> 1) & 1u);
            if (internal) {
                double t;
                if (slab_hit_d(o, dinv, &b->boxes[ci], &t) && t < best && top < 256) stack[top++] = ci;
            } else {
                double t, u, v;
                if (mt_hit_d(o, d, &b->tris[ci], &u, &v, &t) && t < best) {
                    best = t; bi = ci; bu = u; bv = v;
                    if (any_hit) { *idx_out = bi; return best; }
                }
            }
        }
    }
    *idx_out = bi; *u_out = bu; *v_out = bv;
    return best;
}

/* surface() in double for the FP64 estimator (same sampler). */
static void surface_d(const oinfo* in, double u, double v, d3* albedo, d3* normal)
{
    *normal = dnorm(dbary(dld(in->v[0].normal), dld(in->v[1].normal), dld(in->v[2].normal), u, v));
    uint32_t ai = in->m.albedo_idx, ni = in->m.normal_idx;
    int ta = ai < g_texture_count, tn = ni < g_texture_count;
    if (!ta) *albedo = dnorm(dbary(dld(in->v[0].color), dld(in->v[1].color), dld(in->v[2].color), u, v));
    if (!ta && !tn) return;
    double w = 1.0 - u - v;
    double tu = in->v[0].uv[0] * w + in->v[1].uv[0] * u + in->v[2].uv[0] * v;
    double tv = in->v[0].uv[1] * w + in->v[1].uv[1] * u + in->v[2].uv[1] * v;
    double s[4];
    if (ta) {
        tex_sample(&g_textures[ai], tu, tv, s);
        *albedo = dmk(s[0], s[1], s[2]);
    }
    if (tn) {
        tex_sample(&g_textures[ni], tu, tv, s);
        d3 tg = dnorm(dbary(dld(in->v[0].tangent), dld(in->v[1].tangent), dld(in->v[2].tangent), u, v));
        d3 bt = dnorm(dbary(dld(in->v[0].bitangent), dld(in->v[1].bitangent), dld(in->v[2].bitangent), u, v));
        *normal = dnorm(dadd(dadd(dmuls(tg, 2 * s[0] - 1), dmuls(bt, 2 * s[1] - 1)), dmuls(*normal, 2 * s[2] - 1)));
    }
}

static d3 path_radiance_d(const oscene* sc, d3 o, d3 d, uint32_t pixel, uint32_t frame)
{
    uint32_t idx; double u = 0, v = 0;
    double t = trace_d(&sc->bvh, o, d, 0, &idx, &u, &v);
    if (idx == INVALID_IDX) return dmk(0, 0, 0);
    const oinfo* in = info_of(sc, idx);
    d3 hit = dadd(dmuls(d, t), o);
    d3 albedo, normal;
    surface_d(in, u, v, &albedo, &normal);
    d3 acc = dmk(0, 0, 0);
    if (emission_sum(&in->m) > 1e-7f) {
        albedo = dmk(1, 1, 1);
        acc = dld(in->m.emission);
    } else {
        d3 L = dmk(0, 0, 0);
        for (uint32_t i = 0; i < sc->light_count; ++i) {
            const olight* l = &sc->lights[i];
            d3 ldir = dld(l->dir);
            uint32_t si; double su, sv;
            double dist = trace_d(&sc->bvh, dsub(hit, dmuls(ldir, 1e-3)), dmuls(ldir, -1.0), 1, &si, &su, &sv);
            if (!(dist < INFINITY)) L = dadd(L, dmuls(dld(l->color), l->intensity));
            d3 half = dmuls(dsub(dmuls(d, -1.0), ldir), 0.5);
            double df = ddot(normal, dmuls(ldir, -1.0)); df = df > 0 ? df : 0;
            d3 col = dmuls(dmul(L, albedo), df);
            double sh = ddot(normal, half); sh = sh > 0 ? sh : 0;
            if (in->m.specularity > 0.0 && df > 0.0) col = dadd(col, dmuls(dmuls(L, 0.5), pow(sh, in->m.specularity)));
            acc = dadd(acc, col);
        }
    }
    d3 absorbed = albedo;
    for (uint32_t i = 0; i < sc->bounces; ++i) {
        d3 ro = dadd(hit, dmuls(normal, 1e-5));
        float u0, u1;
        cpt_rng_bounce_uniforms(sc->k0, sc->k1, pixel, frame, i, sc->camera, &u0, &u1);
        double rx = u0, ry = u1;
        if (sc->stratified && i == 0) {
            uint32_t pos = frame % 64u;
            rx = ((double)(pos % 8u) + u0) / 8.0;
            ry = ((double)(pos / 8u) + u1) / 8.0;
        }
        double r = sqrt(rx), th = 2.0 * M_PI * ry;
        d3 loc = dmk(r * cos(th), r * sin(th), sqrt(1.0 - rx));
        d3 ax = fabs(normal.x) < FLT_EPSILON ? dcross(normal, dmk(1, 0, 0)) : dcross(normal, dmk(0, 1, 0));
        ax = dnorm(ax);
        d3 ay = dnorm(dcross(normal, ax));
        d3 rd = dadd(dadd(dmuls(ax, loc.x), dmuls(ay, loc.y)), dmuls(normal, loc.z));
        t = trace_d(&sc->bvh, ro, rd, 0, &idx, &u, &v);
        if (idx == INVALID_IDX) break;
        hit = dadd(dmuls(rd, t), ro);
        in = info_of(sc, idx);
        surface_d(in, u, v, &albedo, &normal);
        d3 L = dmk(0, 0, 0);
        if (emission_sum(&in->m) > 1e-7f) {
            double c = -ddot(rd, normal);
            L = dmuls(dld(in->m.emission), c > 0 ? c : 0);
            albedo = dmk(1, 1, 1);
        } else {
            for (uint32_t l = 0; l < sc->light_count; ++l) {
                const olight* li = &sc->lights[l];
                d3 ldir = dld(li->dir);
                uint32_t si; double su, sv;
                double dist = trace_d(&sc->bvh, dsub(hit, dmuls(ldir, 1e-3)), dmuls(ldir, -1.0), 1, &si, &su, &sv);
                double c = -ddot(ldir, normal);
                if (!(dist < INFINITY)) L = dadd(L, dmuls(dmuls(dld(li->color), li->intensity), c > 0 ? c : 0));
            }
        }
        absorbed = dmul(absorbed, albedo);
        acc = dadd(acc, dmuls(dmul(absorbed, L), sc->intensity));
    }
    return acc;
}

/* FP64 estimator: mean radiance per pixel (3 doubles) over spp samples, corner
 * directions as orc_render. */
void orc_render_f64(const otri* sorted, const uint32_t* children, const obox* boxes, uint32_t n,
                    const oinfo* infos, const olight* lights, uint32_t light_count, uint32_t width, uint32_t height,
                    uint32_t spp, uint32_t frame0, uint32_t bounces, float intensity, int stratified, uint32_t k0,
                    uint32_t k1, const ocam* cam, double* mean_out)
{
    oscene sc = {{sorted, children, boxes, n}, infos, lights, light_count, bounces, intensity, stratified, k0, k1,
                 0u};
    memset(mean_out, 0, sizeof(double) * 3 * (size_t)width * height);
    for (uint32_t s = 0; s < spp; ++s) {
        float dirs[4][3];
        orc_corner_dirs(cam, k0, k1, frame0 + s, dirs);
        d3 c00 = dld(dirs[0]), c10 = dld(dirs[1]), c11 = dld(dirs[2]), c01 = dld(dirs[3]), eye = dld(cam->eye);
#pragma omp parallel for schedule(dynamic, 64)
        for (long q = 0; q < (long)width * height; ++q) {
            uint32_t x = (uint32_t)(q % width), y = (uint32_t)(q / width);
            double tx = (double)x / width, ty = (double)y / height;
            d3 a = dadd(c00, dmuls(dsub(c10, c00), tx)), b = dadd(c01, dmuls(dsub(c11, c01), tx));
            d3 dir = dadd(a, dmuls(dsub(b, a), ty));
            d3 r = path_radiance_d(&sc, eye, dir, (uint32_t)q, frame0 + s);
            double* o = mean_out + 3 * q;
            o[0] += r.x; o[1] += r.y; o[2] += r.z;
        }
    }
    for (size_t i = 0; i < 3 * (size_t)width * height; ++i) mean_out[i] /= spp;
}

/* Heat map (visualization.h:19-66): per pixel, base added once per internal box
 * hit, walking every hit box; stops when the 64-entry stack is full. */
void orc_heatmap(const uint32_t* children, const obox* boxes, const ocam* cam, uint32_t width, uint32_t height,
                 const float base[3], float* rgba, uint32_t* counts)
{
    v3 d00 = ld3(cam->dirs[0]), d10 = ld3(cam->dirs[1]), d11 = ld3(cam->dirs[2]), d01 = ld3(cam->dirs[3]);
    v3 eye = ld3(cam->eye);
#pragma omp parallel for schedule(dynamic, 64)
    for (long q = 0; q < (long)width * height; ++q) {
        uint32_t x = (uint32_t)(q % width), y = (uint32_t)(q / width);
        float tx = (float)x / (float)width, ty = (float)y / (float)height;
        v3 dir = mix3(mix3(d00, d10, tx), mix3(d01, d11, tx), ty);
        v3 dinv = mk(1.0f / dir.x, 1.0f / dir.y, 1.0f / dir.z);
        uint32_t stack[STACK_CAP];
        int top = 0, full = 0;
        stack[top++] = 0;
        float a[3] = {0.f, 0.f, 0.f};
        uint32_t count = 0;
        while (top > 0 && !full) {
            uint32_t node = children[stack[--top]];
            for (int side = 0; side < 2 && !full; ++side) {
                if (!((node >> side) & 1u)) continue;
                uint32_t c = (node >> 2) + (uint32_t)side;
                float t;
                if (slab_hit(eye, dinv, &boxes[c], &t)) {
                    stack[top++] = c;
                    for (int k = 0; k < 3; ++k) a[k] = a[k] + base[k];
                    ++count;
                }
                full = top == STACK_CAP;
            }
        }
        rgba[4 * q] = a[0]; rgba[4 * q + 1] = a[1]; rgba[4 * q + 2] = a[2]; rgba[4 * q + 3] = 1.0f;
        if (counts) counts[q] = count;
    }
}

/* Philox known-answer access for the tests. */
void orc_philox(const uint32_t ctr[4], uint32_t k0, uint32_t k1, uint32_t out[4]) { cpt_philox4x32_10(ctr, k0, k1, out); }
void orc_sincos_turns(const float* u, uint32_t m, float* s, float* c)
{
    for (uint32_t i = 0; i < m; ++i) cpt_sincos_turns(u[i], &s[i], &c[i]);
}
