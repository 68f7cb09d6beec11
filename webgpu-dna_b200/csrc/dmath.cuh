// dmath.cuh -- elementary functions and Philox streams of the CUDA path.
//
// The reference computes transport in WGSL (log/exp/sin/cos/pow precision is
// implementation defined) and IRT in JavaScript (Math.*), so neither can be
// reproduced bit for bit.  This library therefore defines its own arithmetic
// for these functions, identical on the GPU and in the CPU oracle:
//
//   log  : x = 2^e m, m in [sqrt(1/2), sqrt 2); s = (m-1)/(m+1);
//          log m = 2 atanh s (Taylor series in s^2, written as fdlibm's
//          f - (f^2/2 - s (f^2/2 + R))), log x = e ln2 + log m.
//   exp  : Cody-Waite reduction x = k ln2 + r, Taylor series of e^r, 2^k scale.
//   sin/cos : reduction by k pi/2 with a three-part constant, Taylor series on
//          [-pi/4, pi/4], quadrant selection.
//
// Split constants of the reductions (hi carries trailing zero bits so that
// k * hi is exact; lo = the constant - hi, rounded):
//   f32 ln2  0x3f317200 + 0x35bfbe8e: fdlibm e_expf.c (Sun Microsystems, 1993)
//   f64 ln2  0x1.62e42fefa3800p-1 + 0x1.ef35793c76730p-45: ARM
//            optimized-routines log_data.c (a 42-bit head)
//   f32 pi/2 1.5703125 + 4.83751297e-4 + 7.54979013e-8: twice DP1..DP3 of
//            Cephes sinf.c (S. L. Moshier)
//   f64 pi/2 pio2_1, pio2_2, pio2_3 of fdlibm e_rem_pio2.c (33 bits each)
// Series coefficients are the exact rationals 1/n! and 1/(2k+1) rounded to the
// working precision.  Error against 40-digit references, over the ranges the
// kernels use: logf, expf, log, exp <= 1 ulp; sin/cos <= 2 ulp (|x| <= 6000
// in f32, 100 in f64); expm1 <= 4 ulp; powf = exp(y ln x) <= 24 ulp for
// y = 1.3 (tests/test_elementary.py, on the oracle's bit-identical copy).
//
// Fused multiply-adds are written explicitly (fmaf/fma); every kernel file is
// compiled with -fmad=false so nothing else is contracted.  Division and sqrt
// are IEEE round-to-nearest (nvcc's default -prec-div/-prec-sqrt).
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
#pragma once
#include <cstdint>


namespace wg {


// ------------------------------------------------------------------ f32 --
__device__ __forceinline__ float logf_(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -__int_as_float(0x7f800000) : __int_as_float(0x7fc00000);
    if (isinf(x)) return x;
    int e = 0;
    uint32_t b = __float_as_uint(x);
    if (b < 0x00800000u) { x = x * 8388608.0f; b = __float_as_uint(x); e = -23; }
    e += (int)(b >> 23) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float f = m - 1.0f;
    float s = f / (2.0f + f);
    float z = s * s;
    float p = fmaf(z, 0.0909090909f, 0.111111111f);
    p = fmaf(z, p, 0.142857143f);
    p = fmaf(z, p, 0.2f);
    p = fmaf(z, p, 0.333333333f);
    p = p * z;
    float hfsq = 0.5f * f * f;
    float lm = f - (hfsq - s * (hfsq + 2.0f * p));
    float fe = (float)e;
    return fmaf(fe, 0.693145752f, fmaf(fe, 1.42860677e-06f, lm));
}

// log of a finite, normal x >= 1e-30 (no special cases; same value as logf_)
__device__ __forceinline__ float logf_pos(float x) {
    uint32_t b = __float_as_uint(x);
    int e = (int)(b >> 23) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421356f) { m = m * 0.5f; e += 1; }
    float f = m - 1.0f;
    float s = f / (2.0f + f);
    float z = s * s;
    float p = fmaf(z, 0.0909090909f, 0.111111111f);
    p = fmaf(z, p, 0.142857143f);
    p = fmaf(z, p, 0.2f);
    p = fmaf(z, p, 0.333333333f);
    p = p * z;
    float hfsq = 0.5f * f * f;
    float lm = f - (hfsq - s * (hfsq + 2.0f * p));
    float fe = (float)e;
    return fmaf(fe, 0.693145752f, fmaf(fe, 1.42860677e-06f, lm));
}

__device__ __forceinline__ float expf_(float x) {
    if (x != x) return x;
    if (x > 88.7228394f) return __int_as_float(0x7f800000);
    if (x < -103.972084f) return 0.0f;
    float kf = rintf(x * 1.44269504f);
    int k = (int)kf;
    float r = fmaf(-kf, 0.693145752f, x);
    r = fmaf(-kf, 1.42860677e-06f, r);
    float p = fmaf(r, 2.48015873e-05f, 1.98412698e-04f);
    p = fmaf(r, p, 1.38888889e-03f);
    p = fmaf(r, p, 8.33333333e-03f);
    p = fmaf(r, p, 4.16666667e-02f);
    p = fmaf(r, p, 1.66666667e-01f);
    p = fmaf(r, p, 0.5f);
    p = fmaf(r, p, 1.0f);
    float y = fmaf(r, p, 1.0f);
    int k1 = k / 2, k2 = k - k1;
    y = y * __uint_as_float((uint32_t)(k1 + 127) << 23);
    y = y * __uint_as_float((uint32_t)(k2 + 127) << 23);
    return y;
}

__device__ __forceinline__ void sincosf_(float x, float* sp, float* cp) {
    float kf = rintf(x * 0.636619747f);
    int q = (int)kf;
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
__device__ __forceinline__ float cosf_(float x) { float s, c; sincosf_(x, &s, &c); return c; }

__device__ __forceinline__ float powf_(float x, float y) {
    if (x == 0.0f) return 0.0f;
    return expf_(y * logf_(x));
}

// ------------------------------------------------------------------ f64 --
__device__ __forceinline__ double log_(double x) {
    if (!(x > 0.0)) return x == 0.0 ? -__longlong_as_double(0x7ff0000000000000ll) : __longlong_as_double(0x7ff8000000000000ll);
    if (isinf(x)) return x;
    int e = 0;
    uint64_t b = (uint64_t)__double_as_longlong(x);
    if (b < 0x0010000000000000ull) { x = x * 4503599627370496.0; b = (uint64_t)__double_as_longlong(x); e = -52; }
    e += (int)(b >> 52) - 1023;
    double m = __longlong_as_double((long long)((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull));
    if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
    double f = m - 1.0;
    double s = f / (2.0 + f);
    double z = s * s;
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
    return fma(fe, 6.93147180559890330187e-01, fma(fe, 5.49792301870837115524e-14, lm));
}

__device__ __forceinline__ double expm1_poly(double r) {
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

__device__ __forceinline__ double scale2(double y, int k) {
    int k1 = k / 2, k2 = k - k1;
    y = y * __longlong_as_double((long long)((uint64_t)(k1 + 1023) << 52));
    y = y * __longlong_as_double((long long)((uint64_t)(k2 + 1023) << 52));
    return y;
}

__device__ __forceinline__ double exp_(double x) {
    if (x != x) return x;
    if (x > 709.782712893384) return __longlong_as_double(0x7ff0000000000000ll);
    if (x < -745.1332191019412) return 0.0;
    double kf = rint(x * 1.4426950408889634);
    int k = (int)kf;
    double r = fma(-kf, 6.93147180559890330187e-01, x);
    r = fma(-kf, 5.49792301870837115524e-14, r);
    double y = 1.0 + expm1_poly(r);
    return scale2(y, k);
}

__device__ __forceinline__ double expm1_(double x) {
    if (fabs(x) <= 0.34657359027997264) return expm1_poly(x);
    return exp_(x) - 1.0;
}

__device__ __forceinline__ double cos_(double x) {
    double kf = rint(x * 0.63661977236758138);
    int q = (int)kf;
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

// --------------------------------------------------------------- Philox --
struct u4 { uint32_t x, y, z, w; };

__device__ __forceinline__ u4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                     uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return u4{c0, c1, c2, c3};
}

// Philox4x32-10 with its round keys supplied (rk[2r], rk[2r+1] = the key of
// round r, as irt.cuh philox_round_keys writes them): the same function as philox()
__device__ __forceinline__ u4 philox_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const uint32_t* rk) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        c0 = hi1 ^ c1 ^ rk[2 * r];
        c1 = lo1;
        c2 = hi0 ^ c3 ^ rk[2 * r + 1];
        c3 = lo0;
    }
    return u4{c0, c1, c2, c3};
}

// u32 -> [0,1] as the reference's rf(): f32(x>>1) / 2147483647.0 == f32(x>>1) * 2^-31
__device__ __forceinline__ float u01f(uint32_t x) { return __uint2float_rn(x >> 1) * 4.65661287e-10f; }
// two words -> double in [0,1) with 53 bits
__device__ __forceinline__ double u01d(uint32_t a, uint32_t b) {
    return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}
// one word -> double in (0,1)
__device__ __forceinline__ double u01d32(uint32_t a) { return ((double)a + 0.5) * (1.0 / 4294967296.0); }
// (a + 1/2) / 2^32 in f32 arithmetic (a truncating conversion and one fma):
// at most 1.5 ulp below and 0.5 ulp above the f32 rounding of u01d32(a), the
// same upward error as that rounding; only for the f32 bounds in front of the
// f64 arithmetic
__device__ __forceinline__ float u01f32(uint32_t a) {
    return fmaf(__uint2float_rz(a), 2.3283064365386963e-10f, 1.1641532182693481e-10f);
}

}  // namespace wg
