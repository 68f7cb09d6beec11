/* oracle/om.h -- elementary functions and random streams of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This header belongs to the CPU oracle that the
 * tests, the smoke check and the benchmark's CPU-baseline leg use to check the
 * CUDA path.  It is never linked into the product library.
 *
 * Why the oracle carries its own elementary functions: the reference computes
 * transport in WGSL, whose log/exp/sin/cos/pow precision is implementation
 * defined, and its IRT in JavaScript (Math.*).  Neither can be reproduced bit
 * for bit, so the product defines one arithmetic for these functions and the
 * oracle restates it independently here:
 *
 *   log  : x = 2^e * m, m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1),
 *          log m = 2 atanh(s) = 2s (1 + s^2/3 + s^4/5 + ...)  (Taylor series
 *          of atanh), log x = e*ln2 + log m with ln2 split in two parts.
 *   exp  : Cody-Waite reduction x = k ln2 + r, |r| <= ln2/2, Taylor series of
 *          e^r, then scaling by 2^k through the exponent bits.
 *   sin/cos : reduction by multiples of pi/2 (three-part Cody-Waite constant),
 *          Taylor series of sin and cos on [-pi/4, pi/4], quadrant selection.
 *
 * Split constants (the head has trailing zero bits so that k * head is exact):
 * f32 ln2 0x3f317200 + 0x35bfbe8e as in fdlibm e_expf.c (Sun, 1993); f64 ln2
 * 0x1.62e42fefa3800p-1 + 0x1.ef35793c76730p-45 as in ARM optimized-routines
 * log_data.c; f32 pi/2 = twice DP1..DP3 of Cephes sinf.c (Moshier); f64 pi/2 =
 * pio2_1..pio2_3 of fdlibm e_rem_pio2.c.  Error bounds in ulps are tested in
 * tests/test_elementary.py through orc_elem (elem.c).
 *
 * Every multiply-add that is fused is written as an explicit fmaf()/fma();
 * the file must be compiled with -ffp-contract=off so that nothing else is
 * fused.  The series coefficients are the exact rationals 1/n! and 1/(2k+1)
 * rounded to the working precision.
 *
 * Random numbers:
 *   - Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 *     easy as 1, 2, 3", SC'11) -- the build's counter-based generator.
 *   - the reference's xoshiro128++-style generator (src/shaders/helpers.wgsl:
 *     188-190) seeded as in src/gpu/buffers.ts:91-104 -- "reference mode".
 */
#ifndef WGDNA_ORACLE_OM_H
#define WGDNA_ORACLE_OM_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline uint32_t om_f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float om_u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint64_t om_d2u(double f) { uint64_t u; memcpy(&u, &f, 8); return u; }
static inline double om_u2d(uint64_t u) { double f; memcpy(&f, &u, 8); return f; }

/* ------------------------------------------------------------------ f32 -- */

/* natural logarithm, x > 0 finite (x <= 0 -> -inf / nan) */
static inline float om_logf(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (isinf(x)) return x;
    int e = 0;
    uint32_t b = om_f2u(x);
    if (b < 0x00800000u) {            /* subnormal: scale by 2^23 */
        x = x * 8388608.0f;
        b = om_f2u(x);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    float m = om_u2f((b & 0x007fffffu) | 0x3f800000u);   /* [1,2) */
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float f = m - 1.0f;
    float s = f / (2.0f + f);
    float z = s * s;
    /* atanh series: R = z/3 + z^2/5 + z^3/7 + z^4/9 + z^5/11 */
    float p = fmaf(z, 0.0909090909f, 0.111111111f);
    p = fmaf(z, p, 0.142857143f);
    p = fmaf(z, p, 0.2f);
    p = fmaf(z, p, 0.333333333f);
    p = p * z;
    /* log m = 2s + 2s*R = f - f*s + 2s*R   (2s = f - f*s) */
    float hfsq = 0.5f * f * f;
    float lm = f - (hfsq - s * (hfsq + 2.0f * p));
    float fe = (float)e;
    return fmaf(fe, 0.693145752f, fmaf(fe, 1.42860677e-06f, lm));
}

/* e^x */
static inline float om_expf(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return INFINITY;
    if (x < -103.972084f) return 0.0f;
    float kf = rintf(x * 1.44269504f);
    int k = (int)kf;
    float r = fmaf(-kf, 0.693145752f, x);
    r = fmaf(-kf, 1.42860677e-06f, r);
    /* e^r - 1 = r + r^2/2 + ... + r^8/8! */
    float p = fmaf(r, 2.48015873e-05f, 1.98412698e-04f);
    p = fmaf(r, p, 1.38888889e-03f);
    p = fmaf(r, p, 8.33333333e-03f);
    p = fmaf(r, p, 4.16666667e-02f);
    p = fmaf(r, p, 1.66666667e-01f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    float y = fmaf(r, p, 1.0f);                    /* e^r in [0.707, 1.414] */
    /* scale by 2^k in two steps so that k down to -150 and up to 128 work */
    int k1 = k / 2, k2 = k - k1;
    y = y * om_u2f((uint32_t)(k1 + 127) << 23);
    y = y * om_u2f((uint32_t)(k2 + 127) << 23);
    return y;
}

/* sin and cos of x (|x| < 2^14) */
static inline void om_sincosf(float x, float *sp, float *cp) {
    float kf = rintf(x * 0.636619747f);
    int q = (int)kf;
    /* pi/2 = 1.5703125 + 4.83751297e-04 + 7.54979013e-08 (3-part split; the
     * first two parts have 11 significant bits, so kf * part is exact) */
    float r = fmaf(-kf, 1.5703125f, x);
    r = fmaf(-kf, 4.83751297e-04f, r);
    r = fmaf(-kf, 7.54979013e-08f, r);
    float z = r * r;
    float s = fmaf(z, 2.75573192e-06f, -1.98412698e-04f);
    s = fmaf(z, s, 8.33333333e-03f);
    s = fmaf(z, s, -1.66666667e-01f);
    s = s * z;
    s = fmaf(r, s, r);
    float c = fmaf(z, -2.75573192e-07f, 2.48015873e-05f);
    c = fmaf(z, c, -1.38888889e-03f);
    c = fmaf(z, c, 4.16666667e-02f);
    c = fmaf(z, c, -0.5f);
    c = fmaf(z, c, 1.0f);
    switch (q & 3) {
    case 0: *sp = s;  *cp = c;  break;
    case 1: *sp = c;  *cp = -s; break;
    case 2: *sp = -s; *cp = -c; break;
    default: *sp = -c; *cp = s; break;
    }
}
static inline float om_cosf(float x) { float s, c; om_sincosf(x, &s, &c); return c; }
static inline float om_sinf(float x) { float s, c; om_sincosf(x, &s, &c); return s; }

/* x^y for x > 0, defined as e^(y log x) */
static inline float om_powf(float x, float y) {
    if (x == 0.0f) return 0.0f;
    return om_expf(y * om_logf(x));
}

/* ------------------------------------------------------------------ f64 -- */

static inline double om_log(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -INFINITY : NAN;
    if (isinf(x)) return x;
    int e = 0;
    uint64_t b = om_d2u(x);
    if (b < 0x0010000000000000ull) {
        x = x * 4503599627370496.0;          /* 2^52 */
        b = om_d2u(x);
        e = -52;
    }
    e += (int)(b >> 52) - 1023;
    double m = om_u2d((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull);
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
    /* R = sum_{k=1..11} z^k/(2k+1) */
    double p = fma(z, 1.0 / 23.0, 1.0 / 21.0);
    p = fma(z, p, 1.0 / 19.0);
    p = fma(z, p, 1.0 / 17.0);
    p = fma(z, p, 1.0 / 15.0);
    p = fma(z, p, 1.0 / 13.0);
    p = fma(z, p, 1.0 / 11.0);
    p = fma(z, p, 1.0 / 9.0);
    p = fma(z, p, 1.0 / 7.0);
    p = fma(z, p, 1.0 / 5.0);
    p = fma(z, p, 1.0 / 3.0);
    p = p * z;
    double hfsq = 0.5 * f * f;
    double lm = f - (hfsq - s * (hfsq + 2.0 * p));
    double fe = (double)e;
    /* ln2 = 6.93147180559890330187e-01 + 5.49792301870837115524e-14 (42-bit head) */
    return fma(fe, 6.93147180559890330187e-01, fma(fe, 5.49792301870837115524e-14, lm));
}

/* e^r - 1 on |r| <= 0.35, Taylor series to r^14 */
static inline double om_expm1_poly(double r) {
    double p = fma(r, 1.0 / 87178291200.0, 1.0 / 6227020800.0);
    p = fma(r, p, 1.0 / 479001600.0);
    p = fma(r, p, 1.0 / 39916800.0);
    p = fma(r, p, 1.0 / 3628800.0);
    p = fma(r, p, 1.0 / 362880.0);
    p = fma(r, p, 1.0 / 40320.0);
    p = fma(r, p, 1.0 / 5040.0);
    p = fma(r, p, 1.0 / 720.0);
    p = fma(r, p, 1.0 / 120.0);
    p = fma(r, p, 1.0 / 24.0);
    p = fma(r, p, 1.0 / 6.0);
    p = fma(r, p, 0.5);
    p = p * r;
    return fma(r, p, r);
}

static inline double om_scale2(double y, int k) {
    int k1 = k / 2, k2 = k - k1;
    y = y * om_u2d((uint64_t)(k1 + 1023) << 52);
    y = y * om_u2d((uint64_t)(k2 + 1023) << 52);
    return y;
}

static inline double om_exp(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return INFINITY;
    if (x < -745.1332191019412) return 0.0;
    double kf = rint(x * 1.4426950408889634);
    int k = (int)kf;
    double r = fma(-kf, 6.93147180559890330187e-01, x);
    r = fma(-kf, 5.49792301870837115524e-14, r);
    double y = 1.0 + om_expm1_poly(r);
    return om_scale2(y, k);
}

/* e^x - 1 */
static inline double om_expm1(double x) {
    if (fabs(x) <= 0.34657359027997264) return om_expm1_poly(x);
    return om_exp(x) - 1.0;
}

/* cos(x), |x| < 2^20 */
static inline double om_cos(double x) {
    double kf = rint(x * 0.63661977236758138);
    int q = (int)kf;
    /* pi/2 split: 1.5707963267341256 + 6.07710050630396597660e-11
     *             + 2.02226624879595063154e-21 (first two parts have 33 bits) */
    double r = fma(-kf, 1.57079632673412561417e+00, x);
    r = fma(-kf, 6.07710050630396597660e-11, r);
    r = fma(-kf, 2.02226624879595063154e-21, r);
    double z = r * r;
    double s = fma(z, -1.0 / 1307674368000.0, 1.0 / 6227020800.0);
    s = fma(z, s, -1.0 / 39916800.0);
    s = fma(z, s, 1.0 / 362880.0);
    s = fma(z, s, -1.0 / 5040.0);
    s = fma(z, s, 1.0 / 120.0);
    s = fma(z, s, -1.0 / 6.0);
    s = s * z;
    s = fma(r, s, r);
    double c = fma(z, 1.0 / 6402373705728000.0, -1.0 / 20922789888000.0);
    c = fma(z, c, 1.0 / 87178291200.0);
    c = fma(z, c, -1.0 / 479001600.0);
    c = fma(z, c, 1.0 / 3628800.0);
    c = fma(z, c, -1.0 / 40320.0);
    c = fma(z, c, 1.0 / 720.0);
    c = fma(z, c, -1.0 / 24.0);
    c = fma(z, c, 0.5);
    c = fma(-z, c, 1.0);
    switch (q & 3) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
    }
}

/* ---------------------------------------------------------------- Philox -- */

typedef struct { uint32_t v[4]; } om_u4;

static inline om_u4 om_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                              uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
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
    om_u4 o = {{c0, c1, c2, c3}};
    return o;
}

/* u32 -> float in [0,1] exactly as the reference's rf():
 *   f32(x >> 1) / 2147483647.0   (helpers.wgsl:190); 2147483647.0 rounds
 *   to 2^31 in f32, so the quotient is f32(x>>1) * 2^-31. */
static inline float om_u01f(uint32_t x) { return (float)(x >> 1) * 4.65661287e-10f; }

/* two u32 -> double in [0,1) with 53 random bits */
static inline double om_u01d(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}
/* one u32 -> double in (0,1) */
static inline double om_u01d32(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }

#endif
