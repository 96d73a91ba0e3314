/*
 * mc3d_exactmath.h -- reproducible single-precision elementary functions.
 *
 * The photon loop of YMC3D (src/mc3d_gpu.cu:74-376) calls logf, acosf, sinf and
 * sincospif.  Vendor implementations of these differ between the host C library
 * and the GPU, so a CPU transcription of the loop cannot follow a GPU trajectory
 * bit for bit.  The functions below are written once, from textbook series, using
 * only IEEE-754 single-precision operations that are correctly rounded on both
 * sides (+, -, *, /, sqrtf, fmaf, floorf).  Compiled with FMA contraction off
 * (gcc -ffp-contract=off, nvcc -fmad=false) they give identical bits on x86-64 and
 * on sm_100a.  The engine's "exact" math mode and the CPU transcription both use
 * them; the engine's "fast" mode uses the GPU's own hardware approximations
 * instead, as the reference does with -use_fast_math (CMakeLists.txt:18).
 *
 * Methods:
 *   logf     : x = 2^e m with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(f/(2+f)),
 *              f = m - 1, atanh Maclaurin series through s^11; ln 2 split into a
 *              12-bit head and a tail (Cody & Waite argument reduction).
 *   sincospi : nearest quarter turn q = floor(2x + 1/2), t = x - q/2 (exact,
 *              |t| <= 1/4); Maclaurin series of sin(pi t) through t^11 and
 *              cos(pi t) through t^12, then a quadrant rotation.
 *   acosf    : c <= 1/2: pi/2 - asin(c); c > 1/2: 2 asin(sqrt((1-c)/2)); asin on
 *              [0, 1/2] by its Maclaurin series sum (2n)!/(4^n n!^2 (2n+1)) y^(2n+1)
 *              through n = 12.
 *   sinf     : Maclaurin series through a^17, for a in [0, pi/2].
 * Every coefficient is the exact series coefficient rounded to float; none is a
 * fitted (minimax) constant.  Accuracy: a few ulp on the stated domains (checked
 * against double-precision libm by the test suite).
 */
#ifndef MC3D_EXACTMATH_H
#define MC3D_EXACTMATH_H

#include <stdint.h>
#include <math.h>
#if !defined(__CUDACC__)
#include <string.h>
#endif

#if defined(__CUDACC__)
#define MC3D_XM_FN static __host__ __device__ __forceinline__
#else
#define MC3D_XM_FN static inline
#endif

MC3D_XM_FN uint32_t mc3d_xm_f2u(float f)
{
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, sizeof u);
    return u;
#endif
}

MC3D_XM_FN float mc3d_xm_u2f(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, sizeof f);
    return f;
#endif
}

/* Natural logarithm of a positive normal float. */
MC3D_XM_FN float mc3d_xm_logf(float x)
{
    uint32_t b = mc3d_xm_f2u(x);
    int e = (int)((b >> 23) & 0xffu) - 127;
    float m = mc3d_xm_u2f((b & 0x007fffffu) | 0x3f800000u); /* [1, 2) */
    if (m > 0x1.6a09e6p+0f) { /* sqrt(2) */
        m = m * 0.5f;
        e += 1;
    }
    float f = m - 1.0f; /* exact (Sterbenz) */
    float s = f / (2.0f + f);
    float z = s * s;
    /* atanh(s)/s - 1 = z/3 + z^2/5 + ... ; Horner from the 1/11 term */
    float p = fmaf(z, 0x1.745d18p-4f /* 1/11 */, 0x1.c71c72p-4f /* 1/9 */);
    p = fmaf(z, p, 0x1.24924ap-3f); /* 1/7 */
    p = fmaf(z, p, 0x1.99999ap-3f); /* 1/5 */
    p = fmaf(z, p, 0x1.555556p-2f); /* 1/3 */
    float t = 2.0f * s;
    float lm = fmaf(t * z, p, t);
    float fe = (float)e;
    /* ln 2 = 0x1.62ep-1 (12 significant bits, so fe * head is exact) + tail */
    return fmaf(fe, 0x1.62e000p-1f, fmaf(fe, 0x1.0bfbe8p-15f, lm));
}

/* sin(pi x) and cos(pi x) for x in [0, 2]. */
MC3D_XM_FN void mc3d_xm_sincospif(float x, float *sp, float *cp)
{
    float q = floorf(2.0f * x + 0.5f);
    float t = x - 0.5f * q; /* exact */
    float z = t * t;
    /* (-1)^n pi^(2n+1) / (2n+1)!, n = 5 .. 0 */
    float s = fmaf(z, -0x1.e30750p-8f, 0x1.507834p-4f);
    s = fmaf(z, s, -0x1.32d2ccp-1f);
    s = fmaf(z, s, 0x1.466bc6p+1f);
    s = fmaf(z, s, -0x1.4abbcep+2f);
    s = fmaf(z, s, 0x1.921fb6p+1f);
    s = s * t;
    /* (-1)^n pi^(2n) / (2n)!, n = 6 .. 0 */
    float c = fmaf(z, 0x1.f9d38ap-10f, -0x1.a6d1f2p-6f);
    c = fmaf(z, c, 0x1.e1f506p-3f);
    c = fmaf(z, c, -0x1.55d3c8p+0f);
    c = fmaf(z, c, 0x1.03c1f0p+2f);
    c = fmaf(z, c, -0x1.3bd3ccp+2f);
    c = fmaf(z, c, 1.0f);
    int quadrant = ((int)q) & 3;
    float so, co;
    switch (quadrant) {
    case 0: so = s; co = c; break;
    case 1: so = c; co = -s; break;
    case 2: so = -s; co = -c; break;
    default: so = -c; co = s; break;
    }
    *sp = so;
    *cp = co;
}

/* asin(y) for y in [0, 1/2]. */
MC3D_XM_FN float mc3d_xm_asin_half(float y)
{
    float z = y * y;
    /* (2n)! / (4^n n!^2 (2n+1)), n = 12 .. 1 */
    float p = fmaf(z, 0x1.a6863ep-8f, 0x1.df3bd4p-8f);
    p = fmaf(z, p, 0x1.12ef3cp-7f);
    p = fmaf(z, p, 0x1.3fde50p-7f);
    p = fmaf(z, p, 0x1.7a8788p-7f);
    p = fmaf(z, p, 0x1.c9999ap-7f);
    p = fmaf(z, p, 0x1.1c4ec4p-6f);
    p = fmaf(z, p, 0x1.6e8ba2p-6f);
    p = fmaf(z, p, 0x1.f1c71cp-6f);
    p = fmaf(z, p, 0x1.6db6dcp-5f);
    p = fmaf(z, p, 0x1.333334p-4f);
    p = fmaf(z, p, 0x1.555556p-3f);
    return fmaf(y * z, p, y);
}

/* acos(c) for c in [0, 1] (NaN propagates). */
MC3D_XM_FN float mc3d_xm_acosf(float c)
{
    if (c <= 0.5f) {
        /* pi/2 = head + tail */
        return (0x1.921fb6p+0f - mc3d_xm_asin_half(c)) + -0x1.777a5cp-25f;
    }
    float y = sqrtf((1.0f - c) * 0.5f);
    return 2.0f * mc3d_xm_asin_half(y);
}

/* sin(a) for a in [0, pi/2] (NaN propagates). */
MC3D_XM_FN float mc3d_xm_sinf(float a)
{
    float z = a * a;
    /* (-1)^n / (2n+1)!, n = 8 .. 1 */
    float p = fmaf(z, 0x1.952c78p-49f, -0x1.ae7f3ep-41f);
    p = fmaf(z, p, 0x1.612462p-33f);
    p = fmaf(z, p, -0x1.ae6456p-26f);
    p = fmaf(z, p, 0x1.71de3ap-19f);
    p = fmaf(z, p, -0x1.a01a02p-13f);
    p = fmaf(z, p, 0x1.111112p-7f);
    p = fmaf(z, p, -0x1.555556p-3f);
    return fmaf(a * z, p, a);
}

#endif /* MC3D_EXACTMATH_H */
