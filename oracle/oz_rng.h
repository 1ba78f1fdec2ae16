/*
 * Oracle — TEST INFRASTRUCTURE ONLY (see walk_oracle.c for the rules of use).
 *
 * Counter-based normal draws, restated independently of the product so that the
 * two can be checked against each other bit for bit:
 *   - Philox4x32-10, from Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
 *     as easy as 1, 2, 3", SC'11 (multipliers, Weyl key increments, 10 rounds);
 *   - Box–Muller (1958) on two 32-bit words;
 *   - ln(m) by the atanh series ln m = 2 atanh((m-1)/(m+1)) after splitting
 *     off the binary exponent, and sin/cos of |y| <= pi/4 by their Taylor series.
 * Every operation is an IEEE single-precision add, multiply, fused multiply-add,
 * divide or square root, or an integer operation, so the same sequence evaluated
 * on a GPU gives the same bits.
 *
 * The reference draws its steps with cuRAND XORWOW + curand_normal
 * (simulation_toolkit/simulation_engine/sim3d_kernel.cu:61-70, :403-405); that
 * generator is not reproduced: parity with the reference is taken with injected
 * draws, statistical otherwise.
 */
#ifndef OZ_RNG_H
#define OZ_RNG_H
#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float oz_bits2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t oz_f2bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* IEEE single constants, given by their bit patterns (value in the comment). */
#define OZ_C_1_3    oz_bits2f(0x3eaaaaabu) /* 1/3 */
#define OZ_C_1_5    oz_bits2f(0x3e4ccccdu) /* 1/5 */
#define OZ_C_1_7    oz_bits2f(0x3e124925u) /* 1/7 */
#define OZ_C_1_9    oz_bits2f(0x3de38e39u) /* 1/9 */
#define OZ_C_LN2    oz_bits2f(0x3f317218u) /* ln 2 */
#define OZ_C_S3     oz_bits2f(0xbe2aaaabu) /* -1/3! */
#define OZ_C_S5     oz_bits2f(0x3c088889u) /* 1/5! */
#define OZ_C_S7     oz_bits2f(0xb9500d01u) /* -1/7! */
#define OZ_C_S9     oz_bits2f(0x3638ef1du) /* 1/9! */
#define OZ_C_C4     oz_bits2f(0x3d2aaaabu) /* 1/4! */
#define OZ_C_C6     oz_bits2f(0xbab60b61u) /* -1/6! */
#define OZ_C_C8     oz_bits2f(0x37d00d01u) /* 1/8! */
#define OZ_C_C10    oz_bits2f(0xb493f27eu) /* -1/10! */
#define OZ_C_HPI    oz_bits2f(0x3fc90fdbu) /* pi/2 */
#define OZ_C_SQRT2  oz_bits2f(0x3fb504f3u) /* sqrt 2 */
#define OZ_C_2M32   oz_bits2f(0x2f800000u) /* 2^-32 */
#define OZ_C_2M33   oz_bits2f(0x2f000000u) /* 2^-33 */
#define OZ_C_2M30   oz_bits2f(0x30800000u) /* 2^-30 */
#define OZ_C_2M24   oz_bits2f(0x33800000u) /* 2^-24 */

/* Philox4x32-10 block: counter (c0..c3), key (k0, k1). */
static inline void oz_philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    uint32_t c0 = c[0], c1 = c[1], c2 = c[2], c3 = c[3];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    c[0] = c0; c[1] = c1; c[2] = c2; c[3] = c3;
}

/* ln x for x in (0, 1], x normal. */
static inline float oz_log_series(float x) {
    uint32_t i = oz_f2bits(x);
    int e = (int)((i >> 23) & 0xffu) - 127;
    float m = oz_bits2f((i & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
    if (m > OZ_C_SQRT2) { m = m * 0.5f; e += 1; }         /* [sqrt(1/2), sqrt(2)] */
    float s = (m - 1.0f) / (m + 1.0f);
    float s2 = s * s;
    float p = fmaf(s2, OZ_C_1_9, OZ_C_1_7);
    p = fmaf(s2, p, OZ_C_1_5);
    p = fmaf(s2, p, OZ_C_1_3);
    p = fmaf(s2, p, 1.0f);
    float lm = (2.0f * s) * p;
    return fmaf((float)e, OZ_C_LN2, lm);
}

/* Two standard normals from two 32-bit words. */
static inline void oz_box_muller(uint32_t ua, uint32_t ub, float* n0, float* n1) {
    float u = fmaf((float)ua, OZ_C_2M32, OZ_C_2M33);          /* (0, 1] */
    float rad = sqrtf(-2.0f * oz_log_series(u));
    uint32_t q = ub >> 30;                                    /* quadrant */
    float t = fmaf((float)(ub & 0x3fffffffu), OZ_C_2M30, -0.5f);
    float y = t * OZ_C_HPI;                                   /* [-pi/4, pi/4] */
    float y2 = y * y;
    float sp = fmaf(y2, OZ_C_S9, OZ_C_S7);
    sp = fmaf(y2, sp, OZ_C_S5);
    sp = fmaf(y2, sp, OZ_C_S3);
    float sn = fmaf(y * y2, sp, y);
    float cp = fmaf(y2, OZ_C_C10, OZ_C_C8);
    cp = fmaf(y2, cp, OZ_C_C6);
    cp = fmaf(y2, cp, OZ_C_C4);
    cp = fmaf(y2, cp, -0.5f);
    float cs = fmaf(y2, cp, 1.0f);
    float c, s;
    switch (q) {
        case 0: c = cs; s = sn; break;
        case 1: c = -sn; s = cs; break;
        case 2: c = -cs; s = -sn; break;
        default: c = sn; s = -cs; break;
    }
    *n0 = rad * c;
    *n1 = rad * s;
}

/* Three normals for draw `draw` of walker `walker` in time step `step`. */
static inline void oz_philox_normal3(uint32_t k0, uint32_t k1, uint32_t stream,
                                     uint32_t walker, uint32_t step, uint32_t draw,
                                     float* n0, float* n1, float* n2) {
    uint32_t c[4] = {walker, step, draw, stream};
    oz_philox4x32_10(c, k0, k1);
    float unused;
    oz_box_muller(c[0], c[1], n0, n1);
    oz_box_muller(c[2], c[3], n2, &unused);
}

/* Three uniforms in [0, 1) for a seeding round (24-bit resolution). */
static inline void oz_philox_uniform3(uint32_t k0, uint32_t k1, uint32_t stream,
                                      uint32_t walker, uint32_t round,
                                      float* u0, float* u1, float* u2) {
    uint32_t c[4] = {walker, round, 0u, stream};
    oz_philox4x32_10(c, k0, k1);
    *u0 = (float)(c[0] >> 8) * OZ_C_2M24;
    *u1 = (float)(c[1] >> 8) * OZ_C_2M24;
    *u2 = (float)(c[2] >> 8) * OZ_C_2M24;
}

#endif
