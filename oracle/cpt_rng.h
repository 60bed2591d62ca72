/* Oracle-side random streams for the path tracer. TEST INFRASTRUCTURE ONLY.
 *
 * The reference draws its path-tracing randoms from curand XORWOW, one state per
 * pixel per frame seeded with host mt19937 output + thread id
 * (cuda_path_tracer.cu:400-402, random.h:13-16), so its images are not
 * reproducible. The rebuild replaces it by design with a counter-based
 * Philox4x32-10 stream (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11), keyed by the render seed, so that the GPU path and
 * this oracle draw identical numbers for the same (pixel, sample, bounce).
 *
 * Stream layout (identical in the product's device code):
 *   bounce i of pixel p, global sample f : counter (p, f, i, c)     -> words 0,1
 *     (c = camera index of a multi-camera render, 0 otherwise)
 *   camera jitter of global sample f     : counter (~0u, f, 0, 1)   -> words 0,1
 *   emitter draw at vertex i (next-event estimation, an extension)
 *                                        : counter (p, f, 0x10000 + i, c) -> words 0,1,2
 *   uniform from a word w                : (w >> 8) * 2^-24, in [0, 1)
 *
 * cpt_sincos_turns(u) returns sin(2*pi*u) and cos(2*pi*u). It replaces the
 * reference's sinf/cosf of CUDA_2PI * u (random.h:97-113) with our own
 * evaluation so that host and device agree to the bit: the argument is reduced
 * exactly in turns (quarter-turn index and the fraction within it, both exact in
 * binary floating point), folded to an eighth of a turn, and sine and cosine of
 * (pi/2)*g, g in [0, 1/2], are evaluated as their Taylor series (sine to degree 9,
 * cosine to degree 10; truncation below 2e-9) in Horner form with fused
 * multiply-adds, which round identically on every IEEE-754 machine.
 */
#ifndef CPT_ORACLE_RNG_H
#define CPT_ORACLE_RNG_H
#include <stdint.h>
#include <math.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline void cpt_philox4x32_10(const uint32_t ctr_in[4], uint32_t k0, uint32_t k1, uint32_t out[4])
{
    /* Multipliers and Weyl key increments from Salmon et al., SC'11, table 2. */
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c0;
        uint64_t p1 = (uint64_t)M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += W0; k1 += W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float cpt_u01(uint32_t w) { return (float)(w >> 8) * (1.0f / 16777216.0f); }

static inline void cpt_rng_bounce_uniforms(uint32_t k0, uint32_t k1, uint32_t pixel, uint32_t sample,
                                           uint32_t bounce, uint32_t camera, float* u0, float* u1)
{
    uint32_t ctr[4] = {pixel, sample, bounce, camera}, o[4];
    cpt_philox4x32_10(ctr, k0, k1, o);
    *u0 = cpt_u01(o[0]);
    *u1 = cpt_u01(o[1]);
}

/* Next-event estimation at vertex `bounce`: counter (p, f, 0x10000 + bounce, c) ->
 * words 0 (emitter), 1, 2 (point on it). */
static inline void cpt_rng_nee_uniforms(uint32_t k0, uint32_t k1, uint32_t pixel, uint32_t sample, uint32_t bounce,
                                        uint32_t camera, float* u0, float* u1, float* u2)
{
    uint32_t ctr[4] = {pixel, sample, 0x10000u + bounce, camera}, o[4];
    cpt_philox4x32_10(ctr, k0, k1, o);
    *u0 = cpt_u01(o[0]);
    *u1 = cpt_u01(o[1]);
    *u2 = cpt_u01(o[2]);
}

static inline void cpt_rng_jitter_uniforms(uint32_t k0, uint32_t k1, uint32_t sample, float* u0, float* u1)
{
    uint32_t ctr[4] = {0xFFFFFFFFu, sample, 0u, 1u}, o[4];
    cpt_philox4x32_10(ctr, k0, k1, o);
    *u0 = cpt_u01(o[0]);
    *u1 = cpt_u01(o[1]);
}

static inline void cpt_sincos_turns(float u, float* s_out, float* c_out)
{
    /* (pi/2)^k / k! rounded to float, signs alternating. */
    /* Written as the exact decimal value of each float so that C and C++14 parse them alike. */
    const float S1 = 1.5707963705062866f, S3 = -0.6459640860557556f, S5 = 0.07969262450933456f,
                S7 = -0.004681753925979137f, S9 = 0.00016044118092395365f;
    const float C2 = -1.2337005138397217f, C4 = 0.25366950035095215f, C6 = -0.020863480865955353f,
                C8 = 0.0009192602592520416f, C10 = -2.520204179745633e-05f;
    float t = u * 4.0f;            /* exact */
    float q = floorf(t);
    float f = t - q;               /* exact, in [0, 1) */
    int quad = ((int)q) & 3;
    int fold = f > 0.5f;
    float g = fold ? 1.0f - f : f; /* exact, in [0, 1/2] */
    float g2 = g * g;
    float sp = fmaf(g2, S9, S7);
    sp = fmaf(g2, sp, S5);
    sp = fmaf(g2, sp, S3);
    sp = fmaf(g2, sp, S1);
    float sg = g * sp;
    float cp = fmaf(g2, C10, C8);
    cp = fmaf(g2, cp, C6);
    cp = fmaf(g2, cp, C4);
    cp = fmaf(g2, cp, C2);
    float cg = fmaf(g2, cp, 1.0f);
    float sa = fold ? cg : sg, ca = fold ? sg : cg;
    float s, c;
    switch (quad) {
        case 0: s = sa; c = ca; break;
        case 1: s = ca; c = -sa; break;
        case 2: s = -sa; c = -ca; break;
        default: s = -ca; c = sa; break;
    }
    *s_out = s;
    *c_out = c;
}

#ifdef __cplusplus
}
#endif
#endif
