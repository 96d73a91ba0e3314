/*
 * mc3d_rng.h -- multiply-with-carry generator and its stream seeding.
 *
 * Generator (gpumcml_rng/gpumcml_rng.cu:38-54): the 64-bit state X packs the
 * carry c in its high word and x in its low word; one draw is
 *     X <- (X mod 2^32) * a + floor(X / 2^32)
 * and returns the low word truncated toward zero to a float (24 significant bits)
 * times 2^-32, a value in [0, 1).  The (0, 1] variant is 1 - that value.
 *
 * Seeding (gpumcml_rng/gpumcml_rng.cu:59-118): line 1 of the safe-prime table is
 * the seeding multiplier `begin`; stream i takes multiplier a_i from the next line
 * and draws (carry, x) from a seeding generator with multiplier `begin`, started at
 * the user seed, retrying while the packed state is invalid.
 *
 * Jump-ahead.  For a state X < m = a 2^32 - 1 one MWC step equals X <- a X mod m
 * (a 2^32 = 1 mod m, so a (c 2^32 + x) = a x + c mod m, and a x + c < m).  The
 * seeding generator after n draws is therefore X0 a^n mod m, which lets every
 * stream compute its own seed independently.  Products mod m use Montgomery
 * reduction with R = 2^64 (m is odd).
 */
#ifndef MC3D_RNG_H
#define MC3D_RNG_H

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define MC3D_RNG_FN static __host__ __device__ __forceinline__
#else
#define MC3D_RNG_FN static inline
#endif

/* unsigned 32-bit integer -> float, rounding toward zero */
MC3D_RNG_FN float mc3d_u32_to_float_rz(uint32_t u)
{
#if defined(__CUDA_ARCH__)
    return __uint2float_rz(u);
#else
    if (u < (1u << 24)) return (float)u;
    int drop = 8 - __builtin_clz(u); /* bits beyond the 24-bit significand */
    return (float)(u & ~((1u << drop) - 1u));
#endif
}

MC3D_RNG_FN uint64_t mc3d_mwc_next(uint64_t x, uint32_t a)
{
    return (x & 0xffffffffull) * (uint64_t)a + (x >> 32);
}

/* [0, 1) */
MC3D_RNG_FN float mc3d_rand_co(uint64_t *x, uint32_t a)
{
    *x = mc3d_mwc_next(*x, a);
    return mc3d_u32_to_float_rz((uint32_t)*x) * 0x1p-32f;
}

/* (0, 1] */
MC3D_RNG_FN float mc3d_rand_oc(uint64_t *x, uint32_t a)
{
    return 1.0f - mc3d_rand_co(x, a);
}

MC3D_RNG_FN uint64_t mc3d_mulhi64(uint64_t a, uint64_t b)
{
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

/* Montgomery product a b R^-1 mod m for a, b < m, m odd, ninv = -m^-1 mod 2^64. */
MC3D_RNG_FN uint64_t mc3d_mont_mul(uint64_t a, uint64_t b, uint64_t m, uint64_t ninv)
{
    uint64_t lo = a * b;
    uint64_t hi = mc3d_mulhi64(a, b);
    uint64_t u = lo * ninv;
    uint64_t um_hi = mc3d_mulhi64(u, m);
    /* lo + u m = 0 mod 2^64, with a carry out unless lo == 0 */
    uint64_t carry = (lo != 0) ? 1u : 0u;
    uint64_t s1 = hi + um_hi;
    uint64_t c1 = (s1 < hi) ? 1u : 0u;
    uint64_t s2 = s1 + carry;
    uint64_t c2 = (s2 < s1) ? 1u : 0u;
    if ((c1 | c2) || s2 >= m) s2 -= m;
    return s2;
}

/* Everything a stream needs to compute its seed: the seeding modulus, its
 * Montgomery constants and, for 4-bit windows w = 0..MC3D_JUMP_WINDOWS-1 and digits
 * d = 1..15, (a^(2 d 16^w) R mod m): the jump by d 16^w seeding attempts (two
 * draws each).  A jump by t < 2^40 attempts is at most ten products. */
#define MC3D_JUMP_BITS 40
#define MC3D_JUMP_WINDOWS (MC3D_JUMP_BITS / 4)
typedef struct {
    uint64_t m;      /* begin * 2^32 - 1 */
    uint64_t ninv;   /* -m^-1 mod 2^64 */
    uint64_t r2;     /* R^2 mod m */
    uint32_t begin;
    uint32_t pad;
    uint64_t jump[MC3D_JUMP_WINDOWS][15];
} mc3d_seed_consts;

/* packed state validity, gpumcml_rng/gpumcml_rng.cu:100 */
MC3D_RNG_FN int mc3d_seed_valid(uint64_t st, uint32_t fora)
{
    return !((st == 0ull) | (((uint32_t)(st >> 32)) >= (fora - 1u)) |
             (((uint32_t)st) >= 0xffffffffu));
}

/* user-seed validity, gpumcml_rng/gpumcml_rng.cu:88 */
MC3D_RNG_FN int mc3d_user_seed_valid(uint64_t xinit, uint32_t begin)
{
    return !((xinit == 0ull) | (((uint32_t)(xinit >> 32)) >= (begin - 1u)) |
             (((uint32_t)xinit) >= 0xffffffffu));
}

/* One seeding attempt from seeding-generator state xs (two draws):
 * gpumcml_rng/gpumcml_rng.cu:103-111.  Returns the packed stream state. */
MC3D_RNG_FN uint64_t mc3d_seed_attempt(uint64_t xs, uint32_t begin, uint32_t fora)
{
    uint64_t x1 = mc3d_mwc_next(xs, begin);
    double frac = (double)((uint32_t)x1) / (double)0x100000000ull;
    uint64_t carry = (uint64_t)(uint32_t)floor(frac * (double)fora);
    uint64_t x2 = mc3d_mwc_next(x1, begin);
    return (carry << 32) + (uint64_t)(uint32_t)x2;
}

/* Seeding-generator state after 2*t draws from xinit (t = attempts so far). */
MC3D_RNG_FN uint64_t mc3d_seed_jump(const mc3d_seed_consts *c, uint64_t xinit, uint64_t t)
{
    uint64_t xm = mc3d_mont_mul(xinit, c->r2, c->m, c->ninv); /* to Montgomery form */
    for (int w = 0; w < MC3D_JUMP_WINDOWS && t != 0; w++, t >>= 4) {
        const unsigned d = (unsigned)(t & 15u);
        if (d) xm = mc3d_mont_mul(xm, c->jump[w][d - 1], c->m, c->ninv);
    }
    return mc3d_mont_mul(xm, 1u, c->m, c->ninv); /* out of Montgomery form */
}

#endif /* MC3D_RNG_H */
