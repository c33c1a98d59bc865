// Elementary functions for the walk-on-spheres kernels, host and device.
//
// Every function here is a short polynomial or series evaluated with explicit
// fmaf(), correctly rounded sqrtf() and IEEE division only.  Compiled with
// contraction disabled (nvcc -fmad=false, g++ -ffp-contract=off) the same
// source gives the same bits on the CPU and on the GPU, which is what lets the
// CUDA walk be compared walk-for-walk against the CPU oracle.
//
// Methods (all from the mathematics, nothing tabulated):
//   * sin/cos on [-pi/4, pi/4]: truncated Maclaurin series, coefficients 1/n!.
//   * sincos of 2*pi*u, u in [0, 1]: exact octant reduction of u, then the
//     series above on the reduced angle.
//   * sin of a general argument: Cody & Waite (1980) additive range reduction
//     by pi/2 split into three float parts, then the series above.
//   * log: x = m * 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
//     s = (m-1)/(m+1), atanh series s + s^3/3 + ... + s^11/11.
//   * exp: x = k ln2 + r (Cody-Waite split of ln2), Maclaurin series of e^r to
//     degree 7, then scaling by 2^k through the exponent bits.
//   * atan2: octant folding to t in [0,1], atan(t) = pi/4 + atan((t-1)/(t+1))
//     for t > tan(pi/8), Maclaurin series of atan to degree 17.
// Accuracy is a few ulp over the ranges the walk uses; the tests measure it
// against the C library in double precision.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define WOS_HD __host__ __device__ __forceinline__
#else
#define WOS_HD inline
#endif

namespace wosm {

// pi and friends, rounded to float from their double values.
static constexpr float kPi     = (float)3.14159265358979323846;
static constexpr float kTwoPi  = (float)6.28318530717958647692;
static constexpr float kInv2Pi = (float)(1.0 / 6.28318530717958647692);
static constexpr float kPiO4   = (float)0.78539816339744830962;

WOS_HD float fabs_(float x) { return fabsf(x); }

// Acceptance test of one bisection step of the largest inscribed ball
// (include/scene.cuh:233-234).  The reference compares the float |d - m|
// with the double literal 1e-5; 1e-5f lies just below 1e-5 and the next float
// above it, so for floats that test is |d - m| <= 1e-5f.
WOS_HD bool ball_accepts(float d, float m) { return fabsf(d - m) <= 1e-5f; }

WOS_HD uint32_t f2u(float x) {
    uint32_t u;
    memcpy(&u, &x, 4);
    return u;
}
WOS_HD float u2f(uint32_t u) {
    float x;
    memcpy(&x, &u, 4);
    return x;
}

// sin(x) for |x| <= pi/4 (a little beyond is fine): x + x^3 * P(x^2).
WOS_HD float sin_poly(float x) {
    const float x2 = x * x;
    float p = (float)(1.0 / 362880.0);
    p = fmaf(p, x2, (float)(-1.0 / 5040.0));
    p = fmaf(p, x2, (float)(1.0 / 120.0));
    p = fmaf(p, x2, (float)(-1.0 / 6.0));
    return fmaf(x * x2, p, x);
}

// cos(x) for |x| <= pi/4: 1 + x^2 * Q(x^2).
WOS_HD float cos_poly(float x) {
    const float x2 = x * x;
    float q = (float)(-1.0 / 3628800.0);
    q = fmaf(q, x2, (float)(1.0 / 40320.0));
    q = fmaf(q, x2, (float)(-1.0 / 720.0));
    q = fmaf(q, x2, (float)(1.0 / 24.0));
    q = fmaf(q, x2, -0.5f);
    return fmaf(x2, q, 1.0f);
}

// (sin, cos) of 2*pi*u for u in [0, 1].  u*8 is exact; its integer part is
// the octant and the fraction is exact as well, so the only rounding before
// the series is the product with pi/4.
WOS_HD void sincos_2pi(float u, float *s, float *c) {
    const float t = u * 8.0f;
    int o = (int)t;
    float f = t - (float)o;
    o &= 7;
    if (o & 1) f = 1.0f - f;
    const float x = f * kPiO4;
    const float sb = sin_poly(x);
    const float cb = cos_poly(x);
    const bool swap = ((o + 1) & 2) != 0;
    float S = swap ? cb : sb;
    float C = swap ? sb : cb;
    if (o & 4) S = -S;
    if ((o + 2) & 4) C = -C;
    *s = S;
    *c = C;
}

// sin(x) for a general finite argument (used by the sinusoid source term).
WOS_HD float sin_(float x) {
    // pi/2 = P1 + P2 + P3, each part a float; P1 has trailing zero bits so
    // k * P1 is exact for |k| < 2^11.
    const float P1 = 1.5703125f;                       // 201/128
    const float P2 = (float)(1.57079632679489661923 - 1.5703125);
    const float P3 = (float)(1.57079632679489661923 - 1.5703125 - (double)(float)(1.57079632679489661923 - 1.5703125));
    const float k = rintf(x * (float)(2.0 / 3.14159265358979323846));
    float r = fmaf(-k, P1, x);
    r = fmaf(-k, P2, r);
    r = fmaf(-k, P3, r);
    const int q = ((int)k) & 3;
    const float s = sin_poly(r);
    const float c = cos_poly(r);
    float v = (q & 1) ? c : s;
    return (q & 2) ? -v : v;
}

WOS_HD float cos_(float x) {
    const float P1 = 1.5703125f;
    const float P2 = (float)(1.57079632679489661923 - 1.5703125);
    const float P3 = (float)(1.57079632679489661923 - 1.5703125 - (double)(float)(1.57079632679489661923 - 1.5703125));
    const float k = rintf(x * (float)(2.0 / 3.14159265358979323846));
    float r = fmaf(-k, P1, x);
    r = fmaf(-k, P2, r);
    r = fmaf(-k, P3, r);
    const int q = ((int)k) & 3;
    const float s = sin_poly(r);
    const float c = cos_poly(r);
    float v = (q & 1) ? s : c;
    return ((q + 1) & 2) ? -v : v;
}

// Natural logarithm for finite x > 0 (x <= 0 gives -inf / NaN).
WOS_HD float log_(float x) {
    if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
    if (x == INFINITY) return x;
    int e = 0;
    if (x < 1.17549435e-38f) {  // subnormal: scale into the normal range
        x *= 8388608.0f;        // 2^23
        e = -23;
    }
    uint32_t b = f2u(x);
    e += (int)((b >> 23) & 0xff) - 127;
    float m = u2f((b & 0x007fffffu) | 0x3f800000u);  // [1, 2)
    if (m > 1.41421356f) {
        m *= 0.5f;
        e += 1;
    }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float q = (float)(1.0 / 11.0);
    q = fmaf(q, z, (float)(1.0 / 9.0));
    q = fmaf(q, z, (float)(1.0 / 7.0));
    q = fmaf(q, z, (float)(1.0 / 5.0));
    q = fmaf(q, z, (float)(1.0 / 3.0));
    const float lm = 2.0f * fmaf(s * z, q, s);
    // ln2 = L1 + L2 with L1 exact in 16 bits so e * L1 is exact.
    const float L1 = 0.693145751953125f;
    const float L2 = (float)(0.69314718055994530942 - 0.693145751953125);
    const float fe = (float)e;
    return fmaf(fe, L1, fmaf(fe, L2, lm));
}

// exp(x) for finite x.
WOS_HD float exp_(float x) {
    if (x > 88.7228394f) return INFINITY;
    if (x < -103.972084f) return 0.0f;
    const float L1 = 0.693145751953125f;
    const float L2 = (float)(0.69314718055994530942 - 0.693145751953125);
    const float k = rintf(x * (float)1.44269504088896340736);
    float r = fmaf(-k, L1, x);
    r = fmaf(-k, L2, r);
    float p = (float)(1.0 / 5040.0);
    p = fmaf(p, r, (float)(1.0 / 720.0));
    p = fmaf(p, r, (float)(1.0 / 120.0));
    p = fmaf(p, r, (float)(1.0 / 24.0));
    p = fmaf(p, r, (float)(1.0 / 6.0));
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    int ki = (int)k;
    // scale by 2^k in two halves so that subnormal results stay correct
    int k1 = ki / 2;
    int k2 = ki - k1;
    const float s1 = u2f((uint32_t)(k1 + 127) << 23);
    const float s2 = u2f((uint32_t)(k2 + 127) << 23);
    return (p * s1) * s2;
}

// atan(t) for t in [0, 1].
WOS_HD float atan01_(float t) {
    float base = 0.0f;
    if (t > 0.41421356f) {  // tan(pi/8)
        t = (t - 1.0f) / (t + 1.0f);
        base = kPiO4;
    }
    const float z = t * t;
    float p = (float)(1.0 / 17.0);
    p = fmaf(p, z, (float)(-1.0 / 15.0));
    p = fmaf(p, z, (float)(1.0 / 13.0));
    p = fmaf(p, z, (float)(-1.0 / 11.0));
    p = fmaf(p, z, (float)(1.0 / 9.0));
    p = fmaf(p, z, (float)(-1.0 / 7.0));
    p = fmaf(p, z, (float)(1.0 / 5.0));
    p = fmaf(p, z, (float)(-1.0 / 3.0));
    return base + fmaf(t * z, p, t);
}

WOS_HD float atan2_(float y, float x) {
    const float ax = fabsf(x), ay = fabsf(y);
    if (ax == 0.0f && ay == 0.0f) return 0.0f;
    const bool swap = ay > ax;
    const float t = swap ? ax / ay : ay / ax;
    float r = atan01_(t);
    if (swap) r = (float)1.57079632679489661923 - r;
    if (x < 0.0f) r = kPi - r;
    return y < 0.0f ? -r : r;
}

// Uniform float in [0, 1) from 32 random bits: the top 23 bits become the
// mantissa of a number in [1, 2), minus one.
WOS_HD float u01(uint32_t x) { return u2f((x >> 9) | 0x3f800000u) - 1.0f; }

}  // namespace wosm
