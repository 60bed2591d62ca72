// Host side of the library: the reference-facing tracer object, synthetic scene
// generators, camera helper and library info.
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <new>
#include <vector>
#include "cpt.h"
#include "cpt_internal.h"
#include "render_hook.h"

namespace cpt {

std::atomic<unsigned long long> g_launches{0};
std::atomic<bool> g_profiling{false};

const char* const kKernelNames[K_KERNEL_COUNT] = {
    "k_bounds", "k_morton", "k_scan_offsets", "k_onesweep", "k_topology", "k_gather_refit", "k_trace",
    "k_generate", "k_extend", "k_shade", "k_wave_counts", "k_accumulate", "k_resolve", "k_ray_sort",
    "k_rc_infer", "k_rc_train", "k_rc_adam", "k_rc_collect", "k_occlude"};

namespace {
struct ProfRecord { int id; cudaEvent_t a, b; };
std::mutex g_prof_mu;
std::vector<ProfRecord> g_prof_records;
std::vector<cudaEvent_t> g_event_pool;
double g_prof_ms[K_KERNEL_COUNT];
double g_prof_busy_ms[K_KERNEL_COUNT];  // union of the launches' intervals (launches on several streams overlap)
unsigned long long g_prof_launches[K_KERNEL_COUNT];

cudaEvent_t take_event()
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    if (!g_event_pool.empty()) {
        cudaEvent_t e = g_event_pool.back();
        g_event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}
}  // namespace

ProfScope::ProfScope(int id_, cudaStream_t s) : id(id_), stream(s)
{
    if (!g_profiling.load(std::memory_order_relaxed)) return;
    start = take_event();
    if (start) cudaEventRecord(start, stream);
}

ProfScope::~ProfScope()
{
    if (!start) return;
    cudaEvent_t stop = take_event();
    if (!stop) return;
    cudaEventRecord(stop, stream);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    g_prof_records.push_back({id, start, stop});
}

int sm_count()
{
    static int cache[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
        cache[dev] = v;
    }
    return cache[dev];
}

// Philox4x32-10 on the host (Salmon et al., SC'11) for the scene generators.
static inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1)
{
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c[0], p1 = (uint64_t)M1 * c[2];
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0; c[1] = (uint32_t)p1; c[2] = n2; c[3] = (uint32_t)p0;
        k0 += W0; k1 += W1;
    }
}
static inline double u01d(uint32_t w) { return (w >> 8) * (1.0 / 16777216.0); }

struct Draw {  // 4 uniforms per counter
    uint32_t seed;
    double u[4];
    void at(uint32_t a, uint32_t b, uint32_t tag)
    {
        uint32_t c[4] = {a, b, tag, 0x5CE7E5u};
        philox(c, seed, 0xA511E9B3u);
        for (int i = 0; i < 4; ++i) u[i] = u01d(c[i]);
    }
};

static void unit_vector(double z01, double phi01, double out[3])
{
    double z = 2.0 * z01 - 1.0, r = sqrt(std::max(0.0, 1.0 - z * z)), ph = 2.0 * M_PI * phi01;
    out[0] = r * cos(ph); out[1] = r * sin(ph); out[2] = z;
}

static void set_tri(cpt_triangle& t, const double* a, const double* b, const double* c, uint32_t info)
{
    for (int k = 0; k < 3; ++k) { t.v0[k] = (float)a[k]; t.v1[k] = (float)b[k]; t.v2[k] = (float)c[k]; }
    t.info_idx = info;
}

// Per-triangle shading record the way extractScene fills it for a mesh without
// normals/colours (PathTracingApp.cpp:49-78): vertex colour = material colour,
// vertex normal = the triangle's geometric normal, no textures.
static void set_info(cpt_triangle_info& in, const cpt_triangle& t, float grey, float emission)
{
    memset(&in, 0, sizeof(in));
    float e1[3], e2[3], n[3];
    for (int k = 0; k < 3; ++k) { e1[k] = t.v1[k] - t.v0[k]; e2[k] = t.v2[k] - t.v0[k]; }
    n[0] = e1[1] * e2[2] - e2[1] * e1[2];
    n[1] = e1[2] * e2[0] - e2[2] * e1[0];
    n[2] = e1[0] * e2[1] - e2[0] * e1[1];
    float len = sqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    float inv = len > 0.f ? 1.0f / len : 0.f;
    for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) {
            in.vertices[v].color[k] = grey;
            in.vertices[v].normal[k] = n[k] * inv;
        }
    for (int k = 0; k < 3; ++k) in.material.emission[k] = emission;
    in.material.specularity = 0.f;
    in.material.albedo_idx = CPT_INVALID_INDEX;
    in.material.normal_map_idx = CPT_INVALID_INDEX;
}

// Emitter quad of side s centred at (cx, y, cz), normal -y.
static uint32_t add_light(cpt_triangle* tris, cpt_triangle_info* infos, uint32_t at, double cx, double y, double cz,
                          double s, float emission)
{
    double h = 0.5 * s;
    double a[3] = {cx - h, y, cz - h}, b[3] = {cx + h, y, cz - h}, c[3] = {cx + h, y, cz + h}, d[3] = {cx - h, y, cz + h};
    set_tri(tris[at], a, b, c, at);
    set_tri(tris[at + 1], a, c, d, at + 1);
    if (infos) {
        for (int k = 0; k < 2; ++k) {
            set_info(infos[at + k], tris[at + k], 1.0f, emission);
            for (int v = 0; v < 3; ++v) {
                infos[at + k].vertices[v].normal[0] = 0.f;
                infos[at + k].vertices[v].normal[1] = -1.f;
                infos[at + k].vertices[v].normal[2] = 0.f;
            }
        }
    }
    return 2;
}

// Value noise on an integer lattice (hashed with Philox), trilinear with a
// smoothstep fade, summed over octaves (fBm).
static double lattice(int64_t x, int64_t y, int64_t z, uint32_t seed)
{
    uint32_t c[4] = {(uint32_t)x, (uint32_t)y, (uint32_t)z, 0xF00Du};
    philox(c, seed, 0x0B5E55EDu);
    return u01d(c[0]) * 2.0 - 1.0;
}
static double value_noise(double x, double y, double z, uint32_t seed)
{
    double fx = floor(x), fy = floor(y), fz = floor(z);
    int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
    double tx = x - fx, ty = y - fy, tz = z - fz;
    tx = tx * tx * (3 - 2 * tx); ty = ty * ty * (3 - 2 * ty); tz = tz * tz * (3 - 2 * tz);
    double c[2][2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int d = 0; d < 2; ++d) c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
    double x00 = c[0][0][0] + tx * (c[1][0][0] - c[0][0][0]), x10 = c[0][1][0] + tx * (c[1][1][0] - c[0][1][0]);
    double x01 = c[0][0][1] + tx * (c[1][0][1] - c[0][0][1]), x11 = c[0][1][1] + tx * (c[1][1][1] - c[0][1][1]);
    double y0 = x00 + ty * (x10 - x00), y1 = x01 + ty * (x11 - x01);
    return y0 + tz * (y1 - y0);
}
static double fbm(double x, double y, double z, uint32_t seed)
{
    double sum = 0, amp = 0.5, freq = 2.0;
    for (int o = 0; o < 6; ++o) {  // 6 octaves, lacunarity 2, gain 0.5
        sum += amp * value_noise(x * freq, y * freq, z * freq, seed + (uint32_t)o);
        freq *= 2.0;
        amp *= 0.5;
    }
    return sum;
}

}  // namespace cpt

using namespace cpt;

extern "C" const char* cpt_version(void) { return "cpt-b200 0.1 (sm_100a)"; }

extern "C" int cpt_profile_begin(void)
{
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (int k = 0; k < K_KERNEL_COUNT; ++k) { g_prof_ms[k] = 0.0; g_prof_busy_ms[k] = 0.0; g_prof_launches[k] = 0; }
    g_profiling.store(true);
    return CPT_OK;
}

extern "C" int cpt_profile_end(void)
{
    g_profiling.store(false);
    std::lock_guard<std::mutex> lk(g_prof_mu);
    int rc = CPT_OK;
    // each launch as an interval on a common time axis (offsets from the first record's
    // start event), then per kernel the length of the union of its intervals
    std::vector<std::pair<double, double>> spans[K_KERNEL_COUNT];
    const cudaEvent_t origin = g_prof_records.empty() ? nullptr : g_prof_records.front().a;
    for (const ProfRecord& r : g_prof_records) {
        float ms = 0.f, t0 = 0.f;
        if (cudaEventSynchronize(r.b) != cudaSuccess || cudaEventElapsedTime(&ms, r.a, r.b) != cudaSuccess ||
            cudaEventElapsedTime(&t0, origin, r.a) != cudaSuccess)
            rc = CPT_ERR_CUDA;
        g_prof_ms[r.id] += ms;
        g_prof_launches[r.id] += 1;
        spans[r.id].push_back({(double)t0, (double)t0 + ms});
    }
    for (int k = 0; k < K_KERNEL_COUNT; ++k) {
        std::sort(spans[k].begin(), spans[k].end());
        double busy = 0.0, a = 0.0, b = -1.0;
        for (const auto& iv : spans[k]) {
            if (iv.first > b) {
                if (b > a) busy += b - a;
                a = iv.first;
                b = iv.second;
            } else if (iv.second > b) {
                b = iv.second;
            }
        }
        if (b > a) busy += b - a;
        g_prof_busy_ms[k] += busy;
    }
    for (const ProfRecord& r : g_prof_records) {
        g_event_pool.push_back(r.a);
        g_event_pool.push_back(r.b);
    }
    g_prof_records.clear();
    return rc;
}

extern "C" int cpt_profile_get(const char* kernel, double* total_ms, unsigned long long* launches)
{
    if (!kernel) return CPT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (int k = 0; k < K_KERNEL_COUNT; ++k)
        if (strcmp(kernel, kKernelNames[k]) == 0) {
            if (total_ms) *total_ms = g_prof_ms[k];
            if (launches) *launches = g_prof_launches[k];
            return CPT_OK;
        }
    return CPT_ERR_INVALID_ARGUMENT;
}
extern "C" int cpt_profile_get_busy(const char* kernel, double* busy_ms)
{
    if (!kernel || !busy_ms) return CPT_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(g_prof_mu);
    for (int k = 0; k < K_KERNEL_COUNT; ++k)
        if (strcmp(kernel, kKernelNames[k]) == 0) {
            *busy_ms = g_prof_busy_ms[k];
            return CPT_OK;
        }
    return CPT_ERR_INVALID_ARGUMENT;
}

extern "C" unsigned long long cpt_launch_count(void) { return g_launches.load(); }

extern "C" uint32_t cpt_scene_random(uint32_t n_random, uint32_t seed, float edge_min, float edge_max, float albedo,
                                     float light_y, float light_size, float light_emission, cpt_triangle* tris,
                                     cpt_triangle_info* infos)
{
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)n_random; ++i) {
        Draw d{seed, {0, 0, 0, 0}};
        d.at((uint32_t)i, 0, 1);
        double c[3] = {d.u[0], d.u[1], d.u[2]};
        double v[3][3];
        for (int k = 0; k < 3; ++k) {
            d.at((uint32_t)i, 1 + (uint32_t)k, 1);
            double len = edge_min + (edge_max - edge_min) * d.u[0], u[3];
            unit_vector(d.u[1], d.u[2], u);
            for (int a = 0; a < 3; ++a) v[k][a] = c[a] + len * u[a];
        }
        set_tri(tris[i], v[0], v[1], v[2], (uint32_t)i);
        if (infos) set_info(infos[i], tris[i], albedo, 0.f);
    }
    uint32_t n = n_random;
    if (light_size > 0.f) n += add_light(tris, infos, n, 0.5, light_y, 0.5, light_size, light_emission);
    return n;
}

extern "C" uint32_t cpt_scene_sphere_hairball(uint32_t nu, uint32_t nv, float amp, uint32_t n_hair, float hair_radius,
                                              uint32_t seed, float albedo, float light_y, float light_size,
                                              float light_emission, cpt_triangle* tris, cpt_triangle_info* infos)
{
    // Lat-long grid: (nu + 1) x (nv + 1) displaced vertices, 2 triangles per quad.
    std::vector<double> pos(3ull * (nu + 1) * (nv + 1));
#pragma omp parallel for schedule(static)
    for (long j = 0; j <= (long)nv; ++j)
        for (uint32_t i = 0; i <= nu; ++i) {
            double th = M_PI * (double)j / nv, ph = 2.0 * M_PI * (double)(i % nu) / nu;
            double dir[3] = {sin(th) * cos(ph), cos(th), sin(th) * sin(ph)};
            double r = 1.0 + amp * fbm(dir[0], dir[1], dir[2], seed);
            double* p = &pos[3 * ((size_t)j * (nu + 1) + i)];
            for (int a = 0; a < 3; ++a) p[a] = r * dir[a];
        }
#pragma omp parallel for schedule(static)
    for (long j = 0; j < (long)nv; ++j)
        for (uint32_t i = 0; i < nu; ++i) {
            const double* a = &pos[3 * ((size_t)j * (nu + 1) + i)];
            const double* b = &pos[3 * ((size_t)j * (nu + 1) + i + 1)];
            const double* c = &pos[3 * ((size_t)(j + 1) * (nu + 1) + i + 1)];
            const double* d = &pos[3 * ((size_t)(j + 1) * (nu + 1) + i)];
            size_t t = 2 * ((size_t)j * nu + i);
            set_tri(tris[t], a, b, c, (uint32_t)t);
            set_tri(tris[t + 1], a, c, d, (uint32_t)(t + 1));
            if (infos) { set_info(infos[t], tris[t], albedo, 0.f); set_info(infos[t + 1], tris[t + 1], albedo, 0.f); }
        }
    const size_t base = 2ull * nu * nv;
    // Hairball: long thin triangles, centres uniform in a ball.
#pragma omp parallel for schedule(static)
    for (long h = 0; h < (long)n_hair; ++h) {
        Draw d{seed ^ 0x4A1Bu, {0, 0, 0, 0}};
        d.at((uint32_t)h, 0, 2);
        double rad = hair_radius * cbrt(d.u[0]), cdir[3];
        unit_vector(d.u[1], d.u[2], cdir);
        double len = 0.05 + 0.15 * d.u[3];
        d.at((uint32_t)h, 1, 2);
        double ax[3];
        unit_vector(d.u[0], d.u[1], ax);
        double width = 1e-4 + 4e-4 * d.u[2];
        double tmp[3] = {fabs(ax[0]) < 0.9 ? 1.0 : 0.0, fabs(ax[0]) < 0.9 ? 0.0 : 1.0, 0.0};
        double bx[3] = {ax[1] * tmp[2] - ax[2] * tmp[1], ax[2] * tmp[0] - ax[0] * tmp[2], ax[0] * tmp[1] - ax[1] * tmp[0]};
        double bl = sqrt(bx[0] * bx[0] + bx[1] * bx[1] + bx[2] * bx[2]);
        double rot = 2.0 * M_PI * d.u[3];
        double cx[3] = {ax[1] * bx[2] - ax[2] * bx[1], ax[2] * bx[0] - ax[0] * bx[2], ax[0] * bx[1] - ax[1] * bx[0]};
        double p0[3], p1[3], p2[3];
        for (int a = 0; a < 3; ++a) {
            double c = rad * cdir[a];
            double w = (cos(rot) * bx[a] + sin(rot) * cx[a]) / bl;
            p0[a] = c - 0.5 * len * ax[a];
            p1[a] = c + 0.5 * len * ax[a];
            p2[a] = c + width * w;
        }
        size_t t = base + (size_t)h;
        set_tri(tris[t], p0, p1, p2, (uint32_t)t);
        if (infos) set_info(infos[t], tris[t], albedo, 0.f);
    }
    uint32_t n = (uint32_t)(base + n_hair);
    if (light_size > 0.f) n += add_light(tris, infos, n, 0.0, light_y, 0.0, light_size, light_emission);
    return n;
}

extern "C" void cpt_scene_bounds(const cpt_triangle* tris, uint32_t n, float out[6])
{
    float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < n; ++i) {
        const float* v[3] = {tris[i].v0, tris[i].v1, tris[i].v2};
        for (int k = 0; k < 3; ++k)
            for (int a = 0; a < 3; ++a) {
                b[a] = v[k][a] < b[a] ? v[k][a] : b[a];          // glm::min: x < y ? x : y
                b[3 + a] = b[3 + a] > v[k][a] ? b[3 + a] : v[k][a]; // glm::max: x > y ? x : y
            }
    }
    memcpy(out, b, sizeof(b));
}

// Column-major 4x4 helpers (glm layout).
static void mat_mul(const double* a, const double* b, double* r)
{
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
            r[c * 4 + rr] = s;
        }
}
static bool mat_inv(const double* m, double* out)
{
    double a[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) { a[r][c] = m[c * 4 + r]; a[r][4 + c] = r == c; }
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r) if (fabs(a[r][c]) > fabs(a[piv][c])) piv = r;
        if (fabs(a[piv][c]) < 1e-300) return false;
        for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
        double d = a[c][c];
        for (int k = 0; k < 8; ++k) a[c][k] /= d;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = a[r][c];
                for (int k = 0; k < 8; ++k) a[r][k] -= f * a[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out[c * 4 + r] = a[r][4 + c];
    return true;
}

extern "C" void cpt_camera_look_at(const float eye[3], const float target[3], const float up[3], float fov_deg,
                                   float aspect, float znear, float zfar, cpt_camera* cam)
{
    // glm::lookAt (right-handed) and glm::perspective (depth -1..1), as the
    // reference's CameraComponent (PathTracingApp.cpp:441).
    double f[3] = {target[0] - (double)eye[0], target[1] - (double)eye[1], target[2] - (double)eye[2]};
    double fl = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    for (int a = 0; a < 3; ++a) f[a] /= fl;
    double s[3] = {f[1] * up[2] - f[2] * up[1], f[2] * up[0] - f[0] * up[2], f[0] * up[1] - f[1] * up[0]};
    double sl = sqrt(s[0] * s[0] + s[1] * s[1] + s[2] * s[2]);
    for (int a = 0; a < 3; ++a) s[a] /= sl;
    double u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2], s[0] * f[1] - s[1] * f[0]};
    double view[16] = {0};
    for (int a = 0; a < 3; ++a) {
        view[a * 4 + 0] = s[a];
        view[a * 4 + 1] = u[a];
        view[a * 4 + 2] = -f[a];
    }
    view[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    view[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    view[14] = (f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]);
    view[15] = 1.0;
    double th = tan(0.5 * fov_deg * M_PI / 180.0);
    double proj[16] = {0};
    proj[0] = 1.0 / (aspect * th);
    proj[5] = 1.0 / th;
    proj[10] = -((double)zfar + znear) / ((double)zfar - znear);
    proj[11] = -1.0;
    proj[14] = -(2.0 * zfar * znear) / ((double)zfar - znear);
    double vp[16], inv[16];
    mat_mul(proj, view, vp);
    mat_inv(vp, inv);
    memset(cam, 0, sizeof(*cam));
    for (int a = 0; a < 3; ++a) cam->eye[a] = eye[a];
    for (int k = 0; k < 16; ++k) cam->inv_view_proj[k] = (float)inv[k];
    // screenToRay of the corners (0,0), (w,0), (w,h), (0,h) at the near plane:
    // NDC (+-1, +-1, -1) -> (+-1, +-1, +1), normalised.
    const double cx[4] = {-1, 1, 1, -1}, cy[4] = {-1, -1, 1, 1};
    for (int c = 0; c < 4; ++c) {
        double ps[4], pe[4];
        for (int r = 0; r < 4; ++r) {
            ps[r] = inv[r] * cx[c] + inv[4 + r] * cy[c] + inv[8 + r] * -1.0 + inv[12 + r];
            pe[r] = inv[r] * cx[c] + inv[4 + r] * cy[c] + inv[8 + r] * 1.0 + inv[12 + r];
        }
        double d[3], l = 0;
        for (int a = 0; a < 3; ++a) { d[a] = pe[a] / pe[3] - ps[a] / ps[3]; l += d[a] * d[a]; }
        l = sqrt(l);
        for (int a = 0; a < 3; ++a) cam->dirs[c][a] = (float)(d[a] / l);
    }
}

// ---------------------------------------------------------------------------
// cpt_tracer: CUDAPathTracer + Scene with caller-free memory management.
// ---------------------------------------------------------------------------
// One uploaded scene with its trees: the triangles, shading records and lights, the
// LBVH and its build scratch, the optional split and wide trees, the emitter table.
// The tracer keeps two: an upload fills the one the current frames do not read, so
// its copies and builds overlap the frames still rendering the other.
struct TracerScene {
    uint32_t n = 0, info_count = 0, light_count = 0;
    void* d_tris = nullptr;
    size_t tris_cap = 0;
    void* d_bvh = nullptr;
    size_t bvh_cap = 0;
    void* d_build_scratch = nullptr;
    size_t build_cap = 0;
    void* d_infos = nullptr;
    size_t infos_cap = 0;
    void* d_lights = nullptr;
    size_t lights_cap = 0;
    void* d_split_nodes = nullptr;  // split traversal BVH (cpt_tracer_set_split)
    size_t split_nodes_cap = 0;
    void* d_split_scratch = nullptr;
    size_t split_scratch_cap = 0;
    void* d_wide_nodes = nullptr;  // compressed wide tree (cpt_tracer_set_wide)
    size_t wide_nodes_cap = 0;
    void* d_wide_tris = nullptr;
    size_t wide_tris_cap = 0;
    void* d_wide_scratch = nullptr;
    size_t wide_scratch_cap = 0;
    void* d_emitters = nullptr;  // emitter table (cpt_tracer_set_nee)
    size_t emitters_cap = 0;
    bool emitters_ready = false;
    cpt_bvh bvh{};
    bool ready = false;
    // built: the trees are complete (build stream); copied: the shading records and
    // lights have landed (copy stream); released: the last frame that read this scene
    // has finished (render stream), so an upload may overwrite it
    cudaEvent_t ev_built = nullptr, ev_copied = nullptr, ev_released = nullptr;
};

struct cpt_tracer {
    int bits = 63;
    cudaStream_t stream = nullptr;        // frames (render, resolve, read-back)
    cudaStream_t build_stream = nullptr;  // triangle uploads and tree builds
    cudaStream_t copy_stream = nullptr;   // shading-record uploads, overlapped with the builds
    int device = 0;
    TracerScene scene[2];
    int front = -1;     // the scene frames render (-1: none uploaded)
    int rendered = -1;  // the scene of the last frame (its status word is the frame's)
    float split_ratio = 0.f;  // 0: traverse the LBVH itself
    uint32_t split_flags = 0;
    uint32_t wide = 0;  // 0 off, 1 the largest-child collapse, 2 the surface-area collapse
    bool nee = false;
    void* d_textures = nullptr;  // cudaTextureObject_t handles (the caller owns the textures)
    size_t textures_cap = 0;
    uint32_t texture_count = 0;
    // frame
    uint32_t width = 0, height = 0;
    void* d_accum = nullptr;
    size_t accum_cap = 0;
    void* d_render_scratch = nullptr;
    size_t render_cap = 0;
    float* d_image = nullptr;
    size_t image_cap = 0;
    unsigned long long* d_counts = nullptr;
    cpt_camera cam{};
    uint32_t frame = 0;
    uint32_t bounces = 1, stratified = 1, seed_lo = 0, seed_hi = 0, accum_mode = CPT_ACCUM_KAHAN;
    float intensity = 3.0f;  // PathTracingSettings.h:26-28 defaults
};

static int ensure(void** p, size_t* cap, size_t bytes)
{
    if (*cap >= bytes && *p) return CPT_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, bytes) != cudaSuccess) { *p = nullptr; return CPT_ERR_CUDA; }
    *cap = bytes;
    return CPT_OK;
}

extern "C" int cpt_tracer_create(cpt_tracer** out, int morton_bits)
{
    if (!out || (morton_bits != 30 && morton_bits != 63)) return CPT_ERR_INVALID_ARGUMENT;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return CPT_ERR_NO_DEVICE;
    cpt_tracer* t = new (std::nothrow) cpt_tracer();
    if (!t) return CPT_ERR_CUDA;
    t->bits = morton_bits;
    cudaGetDevice(&t->device);
    // the build stream at the highest priority: its blocks take the SMs that a frame's
    // launches leave idle (each traversal launch ends on a few long rays) first
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    bool ok = cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithPriority(&t->build_stream, cudaStreamNonBlocking, greatest) == cudaSuccess &&
              cudaStreamCreateWithFlags(&t->copy_stream, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(reinterpret_cast<void**>(&t->d_counts), CPT_RAY_COUNTS * sizeof(unsigned long long)) ==
                  cudaSuccess;
    for (TracerScene& sc : t->scene)
        ok = ok && cudaEventCreateWithFlags(&sc.ev_built, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&sc.ev_copied, cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&sc.ev_released, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        cpt_tracer_destroy(t);
        return CPT_ERR_CUDA;
    }
    cudaMemsetAsync(t->d_counts, 0, CPT_RAY_COUNTS * sizeof(unsigned long long), t->stream);
    *out = t;
    return CPT_OK;
}

extern "C" void cpt_tracer_destroy(cpt_tracer* t)
{
    if (!t) return;
    // every stream may still use the buffers (uploads, builds, frames)
    for (cudaStream_t st : {t->stream, t->build_stream, t->copy_stream})
        if (st) cudaStreamSynchronize(st);
    for (TracerScene& sc : t->scene) {
        void* bufs[] = {sc.d_tris, sc.d_bvh, sc.d_build_scratch, sc.d_infos, sc.d_lights, sc.d_split_nodes,
                        sc.d_split_scratch, sc.d_emitters, sc.d_wide_nodes, sc.d_wide_tris, sc.d_wide_scratch};
        for (void* b : bufs)
            if (b) cudaFree(b);
        for (cudaEvent_t e : {sc.ev_built, sc.ev_copied, sc.ev_released})
            if (e) cudaEventDestroy(e);
    }
    void* bufs[] = {t->d_textures, t->d_accum, t->d_render_scratch, t->d_image, t->d_counts};
    for (void* b : bufs)
        if (b) cudaFree(b);
    for (cudaStream_t st : {t->copy_stream, t->build_stream, t->stream})
        if (st) cudaStreamDestroy(st);
    delete t;
}

extern "C" int cpt_tracer_upload(cpt_tracer* t, const cpt_triangle* tris, uint32_t n, const cpt_triangle_info* infos,
                                 uint32_t info_count, const cpt_dir_light* lights, uint32_t light_count,
                                 const float* enclosing_box)
{
    CPT_RANGE("cpt_tracer_upload");
    if (!t || !tris || !infos || n < 2 || n > kMaxTriangles || info_count == 0 || (light_count && !lights))
        return CPT_ERR_INVALID_ARGUMENT;
    // The scene the frames do not read; its buffers are reused once the last frame that
    // read it has finished (the build and copy streams wait for that, the host does not).
    const int b = t->front < 0 ? 0 : 1 - t->front;
    TracerScene& S = t->scene[b];
    S.ready = false;  // until this upload has queued its builds
    t->front = -1;    // the upload replaces the scene: until it succeeds there is none to render
    int rc;
    if ((rc = ensure(&S.d_tris, &S.tris_cap, sizeof(cpt_triangle) * (size_t)n))) return rc;
    const size_t bvh_bytes = cpt_bvh_bytes(n, t->bits), scr = cpt_lbvh_scratch_bytes(n, t->bits);
    if ((rc = ensure(&S.d_bvh, &S.bvh_cap, bvh_bytes))) return rc;
    if ((rc = ensure(&S.d_build_scratch, &S.build_cap, scr))) return rc;
    if ((rc = ensure(&S.d_infos, &S.infos_cap, sizeof(cpt_triangle_info) * (size_t)info_count))) return rc;
    if (light_count && (rc = ensure(&S.d_lights, &S.lights_cap, sizeof(cpt_dir_light) * (size_t)light_count))) return rc;
    CPT_CUDA_TRY(cudaStreamWaitEvent(t->build_stream, S.ev_released, 0));
    CPT_CUDA_TRY(cudaStreamWaitEvent(t->copy_stream, S.ev_released, 0));
    if ((rc = cpt_bvh_bind(S.d_bvh, S.bvh_cap, n, t->bits, &S.bvh))) return rc;
    // The triangles go first on the build stream (the builds read them); the shading
    // records and lights, which only the renderer reads, go on the copy stream and
    // overlap the builds; the next frame's first shading launch waits for them.
    CPT_CUDA_TRY(cudaMemcpyAsync(S.d_tris, tris, sizeof(cpt_triangle) * (size_t)n, cudaMemcpyHostToDevice,
                                 t->build_stream));
    CPT_CUDA_TRY(cudaMemcpyAsync(S.d_infos, infos, sizeof(cpt_triangle_info) * (size_t)info_count,
                                 cudaMemcpyHostToDevice, t->copy_stream));
    if (light_count)
        CPT_CUDA_TRY(cudaMemcpyAsync(S.d_lights, lights, sizeof(cpt_dir_light) * (size_t)light_count,
                                     cudaMemcpyHostToDevice, t->copy_stream));
    CPT_CUDA_TRY(cudaEventRecord(S.ev_copied, t->copy_stream));
    rc = cpt_lbvh_build(static_cast<const cpt_triangle*>(S.d_tris), n, enclosing_box, t->bits, &S.bvh,
                        S.d_build_scratch, S.build_cap, 0, t->build_stream);
    if (rc) return rc;
    if (t->split_ratio > 0.f) {
        size_t nb = 0;
        const size_t sb = cpt_lbvh_split_bytes(n, t->bits, t->split_ratio, t->split_flags, &nb);
        if (!sb) return CPT_ERR_INVALID_ARGUMENT;
        if ((rc = ensure(&S.d_split_nodes, &S.split_nodes_cap, nb))) return rc;
        if ((rc = ensure(&S.d_split_scratch, &S.split_scratch_cap, sb))) return rc;
        rc = cpt_lbvh_split(&S.bvh, t->split_ratio, t->split_flags, S.d_split_nodes, S.split_nodes_cap,
                            S.d_split_scratch, S.split_scratch_cap, t->build_stream);
        if (rc) return rc;
    }
    if (t->wide) {
        const uint32_t leaves = S.bvh.split_nodes ? S.bvh.split_capacity : n;
        size_t nb = 0, tb = 0;
        const uint32_t wflags = t->wide == 2 ? CPT_WIDE_SAH : 0u;
        const size_t sb = cpt_lbvh_wide_bytes(leaves, wflags, &nb, &tb);
        if (!sb) return CPT_ERR_INVALID_ARGUMENT;
        if ((rc = ensure(&S.d_wide_nodes, &S.wide_nodes_cap, nb))) return rc;
        if ((rc = ensure(&S.d_wide_tris, &S.wide_tris_cap, tb))) return rc;
        if ((rc = ensure(&S.d_wide_scratch, &S.wide_scratch_cap, sb))) return rc;
        rc = cpt_lbvh_wide(&S.bvh, wflags, S.d_wide_nodes, S.wide_nodes_cap, S.d_wide_tris, S.wide_tris_cap,
                           S.d_wide_scratch, S.wide_scratch_cap, t->build_stream);
        if (rc) return rc;
    }
    CPT_CUDA_TRY(cudaEventRecord(S.ev_built, t->build_stream));
    S.n = n;
    S.info_count = info_count;
    S.light_count = light_count;
    S.ready = true;
    S.emitters_ready = false;
    t->front = b;
    t->frame = 0;  // CUDAPathTracer::upload resets the frame counter (cuda_path_tracer.cu:469)
    CPT_CUDA_TRY(cudaMemsetAsync(t->d_counts, 0, CPT_RAY_COUNTS * sizeof(unsigned long long), t->stream));
    return CPT_OK;
}

extern "C" int cpt_tracer_set_split(cpt_tracer* t, float extra_ratio, uint32_t flags)
{
    if (!t || !(extra_ratio >= 0.f) || !(extra_ratio <= 64.f)) return CPT_ERR_INVALID_ARGUMENT;
    if (flags & ~CPT_SPLIT_TREELET) return CPT_ERR_INVALID_ARGUMENT;
    t->split_ratio = extra_ratio;
    t->split_flags = flags;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_wide(cpt_tracer* t, uint32_t on)
{
    if (!t || on > 2) return CPT_ERR_INVALID_ARGUMENT;
    t->wide = on;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_nee(cpt_tracer* t, uint32_t on)
{
    if (!t || on > 1) return CPT_ERR_INVALID_ARGUMENT;
    if ((on != 0) != t->nee) t->frame = 0;  // another estimator: start the accumulation again
    t->nee = on != 0;
    return CPT_OK;
}

// The emitter table of the uploaded scene, sized by a first count (synchronizes once per upload).
static int tracer_emitters(cpt_tracer* t, TracerScene& S, const cpt_scene& sc)
{
    if (S.emitters_ready) return CPT_OK;
    uint32_t cap = 1024, found = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int rc = ensure(&S.d_emitters, &S.emitters_cap, cpt_emitters_bytes(S.n, cap));
        if (rc) return rc;
        rc = cpt_emitters_build(&S.bvh, &sc, cap, S.d_emitters, S.emitters_cap, &found, t->stream);
        if (rc == CPT_OK) {
            S.emitters_ready = true;
            return CPT_OK;
        }
        if (rc != CPT_ERR_SCRATCH_TOO_SMALL) return rc;
        cap = found;
    }
    return CPT_ERR_SCRATCH_TOO_SMALL;
}

extern "C" int cpt_tracer_upload_textures(cpt_tracer* t, const cudaTextureObject_t* textures, uint32_t count)
{
    if (!t || (count && !textures)) return CPT_ERR_INVALID_ARGUMENT;
    int rc;
    if (count && (rc = ensure(&t->d_textures, &t->textures_cap, sizeof(cudaTextureObject_t) * (size_t)count))) return rc;
    if (count)
        CPT_CUDA_TRY(cudaMemcpyAsync(t->d_textures, textures, sizeof(cudaTextureObject_t) * (size_t)count,
                                     cudaMemcpyHostToDevice, t->stream));
    // The host copy may go away when this returns: wait for the copy.
    CPT_CUDA_TRY(cudaStreamSynchronize(t->stream));
    t->texture_count = count;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_primary_rays(cpt_tracer* t, const float dirs[12])
{
    if (!t || !dirs) return CPT_ERR_INVALID_ARGUMENT;
    for (int c = 0; c < 4; ++c)
        for (int a = 0; a < 3; ++a) t->cam.dirs[c][a] = dirs[3 * c + a];
    t->cam.jitter = 0;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_eye(cpt_tracer* t, const float eye[3])
{
    if (!t || !eye) return CPT_ERR_INVALID_ARGUMENT;
    for (int a = 0; a < 3; ++a) t->cam.eye[a] = eye[a];
    return CPT_OK;
}

extern "C" int cpt_tracer_set_camera(cpt_tracer* t, const cpt_camera* cam)
{
    if (!t || !cam) return CPT_ERR_INVALID_ARGUMENT;
    t->cam = *cam;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_settings(cpt_tracer* t, uint32_t bounces, float indirect_intensity, uint32_t stratified,
                                       uint32_t seed_lo, uint32_t seed_hi, uint32_t accum_mode)
{
    if (!t || accum_mode > CPT_ACCUM_F64) return CPT_ERR_INVALID_ARGUMENT;
    if (accum_mode != t->accum_mode) t->frame = 0;
    t->bounces = bounces;
    t->intensity = indirect_intensity;
    t->stratified = stratified;
    t->seed_lo = seed_lo;
    t->seed_hi = seed_hi;
    t->accum_mode = accum_mode;
    return CPT_OK;
}

extern "C" int cpt_tracer_raytrace(cpt_tracer* t, uint32_t width, uint32_t height, uint32_t spp)
{
    CPT_RANGE("cpt_tracer_raytrace");
    if (!t || t->front < 0 || !t->scene[t->front].ready || width == 0 || height == 0 || spp == 0)
        return CPT_ERR_INVALID_ARGUMENT;
    TracerScene& S = t->scene[t->front];
    cpt_render_params p{};
    p.width = width;
    p.height = height;
    p.spp = spp;
    p.frame0 = t->frame;
    p.bounces = t->bounces;
    p.indirect_intensity = t->intensity;
    p.stratified = t->stratified;
    p.seed_lo = t->seed_lo;
    p.seed_hi = t->seed_hi;
    p.accum_mode = t->accum_mode;
    p.nee = t->nee ? 1u : 0u;
    int rc;
    const size_t ab = cpt_accum_bytes(width, height, t->accum_mode), sb = cpt_render_scratch_bytes(&p);
    if (!sb) return CPT_ERR_INVALID_ARGUMENT;
    if (width != t->width || height != t->height) t->frame = p.frame0 = 0;
    // A failed allocation (ensure frees the old buffer first) leaves no image: the
    // next raytrace then starts from frame 0 on a zeroed accumulator.
    if ((rc = ensure(&t->d_accum, &t->accum_cap, ab)) || (rc = ensure(&t->d_render_scratch, &t->render_cap, sb))) {
        t->frame = 0;
        t->width = t->height = 0;
        return rc;
    }
    t->width = width;
    t->height = height;
    if (t->frame == 0) CPT_CUDA_TRY(cudaMemsetAsync(t->d_accum, 0, ab, t->stream));
    CPT_CUDA_TRY(cudaStreamWaitEvent(t->stream, S.ev_built, 0));  // the scene's trees
    cpt_scene sc{static_cast<const cpt_triangle_info*>(S.d_infos), S.info_count,
                 static_cast<const cpt_dir_light*>(S.d_lights), S.light_count,
                 t->texture_count ? static_cast<const cudaTextureObject_t*>(t->d_textures) : nullptr, t->texture_count,
                 nullptr};
    if (t->nee) {
        CPT_CUDA_TRY(cudaStreamWaitEvent(t->stream, S.ev_copied, 0));  // the table reads the shading records
        if ((rc = tracer_emitters(t, S, sc))) return rc;
        sc.emitters = S.d_emitters;
    }
    // the shading records of the last upload may still be copying: the frame's first
    // shading launch waits for them, the primary traversal does not
    cpt_view view{};
    view.bvh = &S.bvh;
    view.scene = &sc;
    view.camera = t->cam;
    view.width = width;
    view.height = height;
    view.accum = t->d_accum;
    RenderHook hook{};
    hook.image_pass = true;
    hook.shade_after = S.ev_copied;
    rc = cpt_render_views_hooked(&view, 1, &p, t->d_render_scratch, t->render_cap, t->d_counts, S.bvh.status, &hook,
                                 t->stream);
    if (rc) return rc;
    CPT_CUDA_TRY(cudaEventRecord(S.ev_released, t->stream));  // the next upload into this scene waits for it
    t->rendered = t->front;
    t->frame += spp;
    return CPT_OK;
}

extern "C" void cpt_tracer_reset_frames(cpt_tracer* t)
{
    if (t) t->frame = 0;
}

extern "C" uint32_t cpt_tracer_frame(const cpt_tracer* t) { return t ? t->frame : 0; }

extern "C" int cpt_tracer_read_image(cpt_tracer* t, float* rgba_host)
{
    CPT_RANGE("cpt_tracer_read_image");
    if (!t || !rgba_host || !t->d_accum || !t->width) return CPT_ERR_INVALID_ARGUMENT;
    int rc;
    const size_t bytes = sizeof(float) * 4 * (size_t)t->width * t->height;
    if ((rc = ensure(reinterpret_cast<void**>(&t->d_image), &t->image_cap, bytes))) return rc;
    if ((rc = cpt_resolve(t->d_accum, t->width, t->height, t->accum_mode, t->d_image, t->stream))) return rc;
    CPT_CUDA_TRY(cudaMemcpyAsync(rgba_host, t->d_image, bytes, cudaMemcpyDeviceToHost, t->stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(t->stream));
    // the status word of the scene the image was rendered from
    return t->rendered < 0 ? CPT_OK : cpt_status_check(t->scene[t->rendered].bvh.status, t->stream);
}

extern "C" int cpt_tracer_resolve(cpt_tracer* t, float* rgba_dev)
{
    CPT_RANGE("cpt_tracer_resolve");
    if (!t || !rgba_dev || !t->d_accum || !t->width || (reinterpret_cast<uintptr_t>(rgba_dev) & 15))
        return CPT_ERR_INVALID_ARGUMENT;
    return cpt_resolve(t->d_accum, t->width, t->height, t->accum_mode, rgba_dev, t->stream);
}

extern "C" int cpt_tracer_get_progress(cpt_tracer* t, void* accum_host, size_t bytes, uint32_t* frame,
                                       uint32_t* accum_mode)
{
    if (!t || !accum_host || !frame || !accum_mode || !t->d_accum || !t->width) return CPT_ERR_INVALID_ARGUMENT;
    if (bytes != cpt_accum_bytes(t->width, t->height, t->accum_mode)) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(accum_host, t->d_accum, bytes, cudaMemcpyDeviceToHost, t->stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(t->stream));
    *frame = t->frame;
    *accum_mode = t->accum_mode;
    return CPT_OK;
}

extern "C" int cpt_tracer_set_progress(cpt_tracer* t, const void* accum_host, size_t bytes, uint32_t width,
                                       uint32_t height, uint32_t frame, uint32_t accum_mode)
{
    if (!t || !accum_host || width == 0 || height == 0) return CPT_ERR_INVALID_ARGUMENT;
    // the Kahan and FP64 layouts have the same size: the mode is checked, not guessed
    if (accum_mode != t->accum_mode) return CPT_ERR_INVALID_ARGUMENT;
    const size_t need = cpt_accum_bytes(width, height, t->accum_mode);
    if (!need || bytes != need) return CPT_ERR_INVALID_ARGUMENT;
    // Until the copy has landed the tracer holds no image: any failure below leaves it
    // to start from frame 0 on a zeroed accumulator at its next raytrace.
    t->frame = 0;
    t->width = t->height = 0;
    int rc;
    if ((rc = ensure(&t->d_accum, &t->accum_cap, need))) return rc;
    CPT_CUDA_TRY(cudaMemcpyAsync(t->d_accum, accum_host, bytes, cudaMemcpyHostToDevice, t->stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(t->stream));  // the host copy may go away
    t->width = width;
    t->height = height;
    t->frame = frame;
    return CPT_OK;
}

extern "C" int cpt_tracer_ray_counts(cpt_tracer* t, unsigned long long out[3])
{
    if (!t || !out) return CPT_ERR_INVALID_ARGUMENT;
    CPT_CUDA_TRY(cudaMemcpyAsync(out, t->d_counts, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, t->stream));
    CPT_CUDA_TRY(cudaStreamSynchronize(t->stream));
    return CPT_OK;
}

extern "C" cudaStream_t cpt_tracer_stream(cpt_tracer* t) { return t ? t->stream : nullptr; }
extern "C" const cpt_bvh* cpt_tracer_bvh(const cpt_tracer* t)
{
    return t && t->front >= 0 ? &t->scene[t->front].bvh : nullptr;
}
