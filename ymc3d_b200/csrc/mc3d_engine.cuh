/*
 * mc3d_engine.cuh -- the photon-tracking hot path on sm_100a.
 *
 * One persistent kernel runs every photon of every job in a launch.  The unit of
 * work is an RNG *stream*: stream i of a job owns multiplier a_(i mod M) of the
 * safe-prime table and runs the job's photons i, i+S, i+2S, ... one after
 * another, continuing the same multiply-with-carry sequence, exactly as one
 * photon slot of the reference does (src/mc3d_gpu.cu:74-111, 128-376) minus the
 * masked steps a frozen slot burns until the next host round trip.  Threads take
 * streams from a global counter, so the trajectories depend on (table, seed,
 * photons, streams) only -- never on the grid shape or on scheduling -- and the
 * tallies, being 64-bit integer sums, are bit-reproducible.
 *
 * Per-step physics follows src/mc3d_gpu.cu:175-340 operation for operation,
 * including its quirks (Fresnel denominator, 0/0 -> transmit at normal incidence,
 * mirror short-circuit after a Fresnel reflection, freeze one step after entering
 * air, i/j/k re-derived from the position every 45 steps, the NaN/db==0 quickfix
 * at the end of each 45-step chunk).  The math policy fixes the transport type
 * and how the elementary operations are evaluated: MathExact uses correctly
 * rounded IEEE operations and the reproducible series of mc3d_exactmath.h
 * (bit-identical to the CPU transcription), MathFast uses the GPU's approximate
 * instructions like the reference's -use_fast_math build, MathF64 steps in FP64.
 * With fast math the face crossings inside cubes of uniform tissue can be merged
 * into one step (photon_step's JUMP).
 */
#ifndef MC3D_ENGINE_CUH
#define MC3D_ENGINE_CUH

#include <stdint.h>
#include <cuda_runtime.h>
#include "mc3d_rng.h"
#include "mc3d_exactmath.h"
#include "mc3d_device_types.h"

namespace mc3d {

/* ---------------------------------------------------------------- math policies
 * A policy fixes the transport arithmetic type (real) and how the elementary
 * operations are evaluated, and reads the per-tissue coefficients of the optical
 * table (three float4 per tissue, see photon_step). */

/* The FP32 policies read every coefficient as the float the reference computes
 * per step, precomputed on the host. */
struct FloatTable {
    using real = float;
    static __device__ __forceinline__ float n(const float4 *tt) { return tt[0].w; }
    static __device__ __forceinline__ float mu_t(const float4 *tt) { return tt[1].x; }
    static __device__ __forceinline__ float albedo_c(const float4 *tt) { return tt[1].y; }
    static __device__ __forceinline__ float rmu_t(const float4 *tt) { return tt[1].z; }
    /* Henyey-Greenstein cos(theta) for the draw xi in (0, 1] (src/mc3d_gpu.cu:282-286) */
    template <class M>
    static __device__ __forceinline__ float hg_cos(const float4 *tt, float xi)
    {
        const float4 t2 = tt[2];
        float c = M::div(t2.x, t2.y + t2.z * xi);
        return tt[1].w * (t2.w - c * c);
    }
    /* thresholds of src/mc3d_types.h:11-18, see the constants below */
    static __device__ __forceinline__ bool w_below_threshold(float w) { return w <= 0x1.a36e2ep-14f; }
    static __device__ __forceinline__ bool uz_within(float u) { return u <= 0x1.fffeb0p-1f; }
    static __device__ __forceinline__ float roulette_survivor(float w)
    {
        return (float)((double)w / 0.1);
    }
    static __device__ __forceinline__ float zero_threshold() { return (float)(1 - 0.99999); }
    /* fixed-point weight, 2^-32 resolution */
    static __device__ __forceinline__ uint64_t qw(float w) { return __float2ull_rn(w * 4294967296.0f); }
};

struct MathExact : FloatTable {
    static constexpr bool kFast = false;
    /* a product rounded on its own, never fused into a following add */
    static __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
    /* a / b where the caller also holds r = 1/b: the exact policy divides */
    static __device__ __forceinline__ float div_r(float a, float b, float) { return a / b; }
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return 1.0f / sqrtf(x); }
    static __device__ __forceinline__ float log(float x) { return mc3d_xm_logf(x); }
    static __device__ __forceinline__ float acos(float x) { return mc3d_xm_acosf(x); }
    static __device__ __forceinline__ float sin(float x) { return mc3d_xm_sinf(x); }
    static __device__ __forceinline__ void sincospi(float x, float *s, float *c)
    {
        mc3d_xm_sincospif(x, s, c);
    }
    static __device__ __forceinline__ float floor(float x) { return floorf(x); }
    static __device__ __forceinline__ float fmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fabs(float x) { return fabsf(x); }
    static __device__ __forceinline__ float copysign(float a, float b) { return copysignf(a, b); }
};

/* Compiled only in a translation unit built with -use_fast_math, where the
 * operators and functions below map to the approximate hardware paths. */
struct MathFast : FloatTable {
    static constexpr bool kFast = true;
    static __device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
    /* every denominator divided here is a direction cosine, a sum of products of
     * cosines and sines, a refractive-index sum or 1 - g + 2 g xi, all far below the
     * 2^126 where __fdividef stops being defined; x / 0 still gives +-inf or NaN */
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float div_r(float a, float, float r) { return a * r; }
    static __device__ __forceinline__ float sqrt(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsqrt(float x) { return rsqrtf(x); }
    static __device__ __forceinline__ float log(float x) { return logf(x); }
    static __device__ __forceinline__ float acos(float x) { return acosf(x); }
    static __device__ __forceinline__ float sin(float x) { return sinf(x); }
    /* sin/cos(pi x) for x in [0, 2): the SFU's sin/cos on pi (x - 1) in [-pi, pi) */
    static __device__ __forceinline__ void sincospi(float x, float *s, float *c)
    {
        float sn, cs;
        __sincosf(3.14159265358979f * (x - 1.0f), &sn, &cs);
        *s = -sn;
        *c = -cs;
    }
    static __device__ __forceinline__ float floor(float x) { return floorf(x); }
    static __device__ __forceinline__ float fmin(float a, float b) { return fminf(a, b); }
    static __device__ __forceinline__ float fabs(float x) { return fabsf(x); }
    static __device__ __forceinline__ float copysign(float a, float b) { return copysignf(a, b); }
};

/* FP64 stepping: the same loop with every transport quantity in double, the
 * coefficients derived in double from the table's float (mua, mus, g, n), and
 * the reference's double literals compared in double.  Random numbers stay the
 * reference's 32-bit draws.  Built with IEEE division and square root; the
 * precision reference for the FP32 policies. */
struct MathF64 {
    using real = double;
    static constexpr bool kFast = false;
    static __device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return a / b; }
    static __device__ __forceinline__ double div_r(double a, double b, double) { return a / b; }
    static __device__ __forceinline__ double sqrt(double x) { return ::sqrt(x); }
    static __device__ __forceinline__ double rsqrt(double x) { return 1.0 / ::sqrt(x); }
    static __device__ __forceinline__ double log(double x) { return ::log(x); }
    static __device__ __forceinline__ double acos(double x) { return ::acos(x); }
    static __device__ __forceinline__ double sin(double x) { return ::sin(x); }
    static __device__ __forceinline__ void sincospi(double x, double *s, double *c)
    {
        ::sincospi(x, s, c);
    }
    static __device__ __forceinline__ double floor(double x) { return ::floor(x); }
    static __device__ __forceinline__ double fmin(double a, double b) { return ::fmin(a, b); }
    static __device__ __forceinline__ double fabs(double x) { return ::fabs(x); }
    static __device__ __forceinline__ double copysign(double a, double b) { return ::copysign(a, b); }
    static __device__ __forceinline__ double n(const float4 *tt) { return tt[0].w; }
    static __device__ __forceinline__ double mu_t(const float4 *tt)
    {
        return (double)tt[0].x + (double)tt[0].y;
    }
    static __device__ __forceinline__ double albedo_c(const float4 *tt)
    {
        return (double)tt[0].x / mu_t(tt);
    }
    static __device__ __forceinline__ double rmu_t(const float4 *tt) { return 1.0 / mu_t(tt); }
    template <class M>
    static __device__ __forceinline__ double hg_cos(const float4 *tt, double xi)
    {
        const double g = tt[0].z;
        const double c = (1 - g * g) / (1 - g + 2 * g * xi);
        return (1 + g * g - c * c) / (2 * g);
    }
    static __device__ __forceinline__ bool w_below_threshold(double w) { return w < 0.0001; }
    static __device__ __forceinline__ bool uz_within(double u) { return u <= 0.99999; }
    static __device__ __forceinline__ double roulette_survivor(double w) { return w / 0.1; }
    static __device__ __forceinline__ double zero_threshold() { return 1 - 0.99999; }
    static __device__ __forceinline__ uint64_t qw(double w)
    {
        return __double2ull_rn(w * 4294967296.0);
    }
};

/* ------------------------------------------------------------ reference constants
 * src/mc3d_types.h:11-18.  SURVIVAL_CHANCE, W_THRESHOLD and UZ_THRESH are double
 * literals there, so a float compared with them is widened to double.  No float
 * lies between each literal and the float bound below, so these float comparisons
 * decide exactly as the double ones do (the unit tests enumerate the neighbours):
 *   (double)e <  0.1      <=>  e <  0x1.99999ap-4f   ((float)0.1 is above 0.1)
 *   (double)w <  0.0001   <=>  w <= 0x1.a36e2ep-14f  ((float)0.0001 is below it)
 *   (double)u <= 0.99999  <=>  u <= 0x1.fffeb0p-1f   ((float)0.99999 is below it)
 * The roulette division W / 0.1 stays in double, as in the reference. */
#define MC3D_SURVIVAL_CHANCE 0.1
#define MC3D_SURVIVAL_LT_F 0x1.99999ap-4f
#define MC3D_W_THRESHOLD_LE_F 0x1.a36e2ep-14f
#define MC3D_UZ_THRESH 0.99999
#define MC3D_UZ_THRESH_LE_F 0x1.fffeb0p-1f
/* fast math: |1 - sin^2(theta_t)| below this takes the FP64 Fresnel branch */
#define MC3D_NEAR_CRITICAL_F 0x1p-5f
#define MC3D_NUM_PHOTON_STEPS 45
#define MC3D_TISSUE_AIR 0
#define MC3D_TAB_STRIDE 3 /* float4 per tissue in the optical table */


/* src/mc3d_gpu.cu:53-63 */
template <class M, class R = typename M::real>
static __device__ __forceinline__ int grid_coord(R x, R ux, float d_, float rd_)
{
    const R d = d_, rd = rd_;
    /* the index is carried as a float (exact for |i| < 2^24), which saves the
     * int <-> float conversions of the two face products */
    R fi = M::floor(M::div_r(x, d, rd));
    const R f1 = fi + (R)1;
    const R hi = f1 * d;
    const bool up = (x == hi);
    fi = up ? f1 : fi;
    const R bmin = up ? hi : fi * d;
    const bool stay = (x > bmin) || ((x == bmin) && (ux >= 0));
    return (int)fi - (stay ? 0 : 1);
}

/* src/mc3d_gpu.cu:24-27 with the clamp addressing of the texture (:416-418).
 * With JUMP the lookup reads the packed map (tissue | box radius << 8, one
 * 16-bit load), so the box radius rides in bits 8-15 of the result (0 above
 * the surface, where the tissue is air). */
template <bool JUMP = false, class R = float>
static __device__ __forceinline__ int tissue_at(const GeomDev &g, int i, int j, int k, R z, R uz)
{
    int ci = min(max(i, 0), g.nx - 1);
    int cj = min(max(j, 0), g.ny - 1);
    int ck = min(max(k, 0), g.nz - 1);
    int t;
    if (JUMP) {
        const int rk = min(max(k, 0), g.nz - 1 + MC3D_SAFE_CAP);
        /* 32-bit index: plans take merged steps only for maps below 2^32 cells */
        t = __ldg(g.cells + (((uint32_t)rk * (uint32_t)g.ny + (uint32_t)cj) * (uint32_t)g.nx +
                             (uint32_t)ci));
    } else {
        t = __ldg(g.tissue + ((int64_t)ck * g.ny + cj) * g.nx + ci);
    }
    return ((z <= 0) && (uz < 0)) ? MC3D_TISSUE_AIR : t;
}

/* src/mc3d_gpu.cu:29-49.  With r > 0 the box is the cube of voxels within
 * Chebyshev distance r of (i, j, k) instead of the voxel itself.  Each border is
 * a rounded product, as the reference's separate multiply gives it: fused into
 * the subtraction that follows (which the compiler may do where the snapped
 * positions are unused), a photon lying exactly on a face would see its
 * distance to that face as the product's rounding error instead of 0. */
template <class M, class R = typename M::real>
static __device__ __forceinline__ R intersection(const GeomDev &g, int i, int j, int k, R *x, R ux,
                                                 R *y, R uy, R *z, R uz, int r = 0)
{
    R border_x = M::mul_rn((R)((ux >= 0) ? (int)((unsigned)i + 1u + r) : i - r), (R)g.dx);
    R t_x = M::div(border_x - *x, ux);
    R border_y = M::mul_rn((R)((uy >= 0) ? (int)((unsigned)j + 1u + r) : j - r), (R)g.dy);
    R t_y = M::div(border_y - *y, uy);
    R border_z = M::mul_rn((R)((uz >= 0) ? (int)((unsigned)k + 1u + r) : k - r), (R)g.dz);
    R t_z = M::div(border_z - *z, uz);
    R t = M::fmin(t_x, M::fmin(t_y, t_z));
    *x = (t == t_x) ? border_x : *x + ux * t;
    *y = (t == t_y) ? border_y : *y + uy * t;
    *z = (t == t_z) ? border_z : *z + uz * t;
    return t;
}

/* src/mc3d_gpu.cu:113-126 */
template <class M, class R = typename M::real>
static __device__ __forceinline__ bool mirror(R *x, R *ux, float length_)
{
    const R length = length_;
    bool refl = (*x >= length) || (*x <= 0);
    *x = (*x >= length) ? 2 * length - *x : *x;
    *x = (*x <= 0) ? M::fabs(*x) : *x;
    *ux = refl ? -1 * (*ux) : *ux;
    return refl;
}

template <class R>
struct PhotonT {
    R x, y, z, ux, uy, uz, W, s;
    int i, j, k, tissue;
};

/* Per-thread tallies live in shared memory, one column per thread, so that the
 * step loop keeps only the photon in registers.  They are touched when a photon
 * ends or at a roulette event, and flushed to the job's totals when the thread
 * moves to another stream.  Slot order is mc3d_totals (include/mc3d.h). */
enum {
    T_PHOTONS = 0, T_STEPS, T_W_LAUNCHED, T_R_IN, T_R_OUT, T_T_IN, T_T_OUT, T_ABSORBED,
    T_RR_KILLED, T_RR_CREATED, T_LOST, T_CAPPED, T_QUICKFIX, T_FRESNEL
};
#define MC3D_MAX_BLOCK 256

struct Acc {
    unsigned long long *col; /* sh_acc + threadIdx.x; slot t at col[t * MC3D_MAX_BLOCK] */
    __device__ __forceinline__ unsigned long long &operator[](int t) const
    {
        return col[t * MC3D_MAX_BLOCK];
    }
};

/* One step of src/mc3d_gpu.cu:175-340 for a live photon.  Returns true when the
 * photon froze during this step; *db receives the step's boundary distance.
 *
 * JUMP (merged steps): p.tissue carries a box radius r in bits 8-15, and the
 * step's box is the cube of voxels within Chebyshev distance r of the photon's
 * voxel.  The box holds only the photon's tissue, and a shell of one voxel around
 * it has the photon's refractive index and stays clear of the top and lateral
 * faces (pack_kernel): a step that reaches a box face crosses into a voxel of the
 * same index, with no Fresnel event, no mirror and no air rule, exactly as the
 * reference's step at that face would (snapped, next voxel by the face rule; that
 * voxel may hold another tissue of the same index, whose coefficients the next
 * step uses).
 * The face crossings inside the box, which in the reference only move the
 * photon (no absorption or scattering; their four random numbers are drawn and
 * discarded), are merged into this one step.  Every reflection therefore
 * happens in a one-voxel step (r = 0), where the reference's rule applies
 * unchanged: a reflected photon keeps the voxel index it started the step with
 * (src/mc3d_gpu.cu:334-339).  That rule can leave the index one voxel off when a
 * coordinate that was not snapped rounded onto a face; the photon then takes
 * zero-length steps until the quickfix at its chunk's end removes it, which is
 * part of the weight the reference loses. */
template <class M, bool AMAP, bool JUMP = false, class R = typename M::real>
static __device__ __forceinline__ bool photon_step(const GeomDev &g, const float4 *tab,
                                                   PhotonT<R> &p, uint64_t &rx, uint32_t ra,
                                                   const Acc &acc, R *db_out,
                                                   uint32_t *fresnel_count,
                                                   unsigned long long *amap, bool *lat_mirror)
{
    /* per tissue: (mua, mus, g, n), (mu_t, mua/mu_t, 1/mu_t, 1/(2g)),
     * (1-g^2, 1-g, 2g, 1+g^2) -- each the float the reference computes per step */
    const int tis = JUMP ? (p.tissue & 0xff) : p.tissue;
    const float4 *tt = tab + MC3D_TAB_STRIDE * tis;
    R ni = M::n(tt);
    R nt = ni;
    const R mu_t = M::mu_t(tt);
    const R rmu_t = M::rmu_t(tt);

    R newx = p.x, newy = p.y, newz = p.z;
    R db = intersection<M>(g, p.i, p.j, p.k, &newx, p.ux, &newy, p.uy, &newz, p.uz,
                               JUMP ? (p.tissue >> 8) : 0);

    bool hit = db * mu_t <= p.s;
    R ds = hit ? db * mu_t : p.s;
    newx = hit ? newx : p.x + M::div_r(p.ux * ds, mu_t, rmu_t);
    newy = hit ? newy : p.y + M::div_r(p.uy * ds, mu_t, rmu_t);
    newz = hit ? newz : p.z + M::div_r(p.uz * ds, mu_t, rmu_t);
    R s = p.s - ds;

    int nexti = grid_coord<M>(newx, p.ux, g.dx, g.rdx);
    int nextj = grid_coord<M>(newy, p.uy, g.dy, g.rdy);
    int nextk = grid_coord<M>(newz, p.uz, g.dz, g.rdz);
    int next_tissue = tissue_at<JUMP>(g, nexti, nextj, nextk, newz, p.uz);
    nt = M::n(tab + MC3D_TAB_STRIDE * (JUMP ? (next_tissue & 0xff) : next_tissue));

    R tr_ux = p.ux, tr_uy = p.uy, tr_uz = p.uz;
    bool refl = false;
    if (ni != nt) { /* src/mc3d_gpu.cu:226-257 */
        R cos_ai = (p.i != nexti) ? p.ux : ((p.j != nextj) ? p.uy : p.uz);
        cos_ai = M::fabs(cos_ai);
        cos_ai = (cos_ai > 1) ? 1 : cos_ai;
        R ni_nt = M::div(ni, nt);
        /* sin(acos(c)); fast math evaluates it as sqrt((1 - c)(1 + c)), the same
         * value without the polynomial of acosf (and more accurate near c = 1) */
        R sin_ai = M::kFast ? M::sqrt(((R)1 - cos_ai) * ((R)1 + cos_ai))
                            : M::sin(M::acos(cos_ai));
        R sin_at = ni_nt * sin_ai;
        R cos_at = M::sqrt((R)1 - sin_at * sin_at);
        R R1 = M::div(sin_ai * cos_at - cos_ai * sin_at, sin_ai * cos_at + cos_ai * sin_at);
        R R2 = M::div(cos_ai * cos_at - sin_ai * sin_at, cos_ai * cos_at + sin_at * sin_at);
        R Rf = 0.5 * R1 * R1 * ((R)1 + R2 * R2); /* 0.5 is a double literal there too */
        Rf = (sin_at > 1) ? 1 : Rf;
        Rf = (ni == nt) ? 0 : Rf;
        R lat = ni_nt; /* scale of the transmitted lateral cosines */
        if (M::kFast && M::fabs((R)1 - sin_at * sin_at) < MC3D_NEAR_CRITICAL_F) {
            /* Near the critical angle 1 - sin_at^2 cancels in float and R is steep:
             * the same formulas in FP64, sin_ai from cos_ai directly, and the
             * transmitted direction renormalised in FP64. */
            const double c = cos_ai;
            const double rn = (double)ni / (double)nt;
            const double si = sqrt((1.0 - c) * (1.0 + c));
            const double st = rn * si;
            const double ca = sqrt(fmax((1.0 - st) * (1.0 + st), 0.0));
            const double R1 = (si * ca - c * st) / (si * ca + c * st);
            const double R2 = (c * ca - si * st) / (c * ca + st * st);
            Rf = (st >= 1.0) ? (R)1 : (R)(0.5 * R1 * R1 * (1.0 + R2 * R2));
            const bool xa = p.i != nexti;
            const bool ya = !xa && p.j != nextj;
            const bool za = !xa && !ya && p.k != nextk;
            const double ax = xa ? 0.0 : (double)p.ux;
            const double ay = ya ? 0.0 : (double)p.uy;
            const double az = za ? 0.0 : (double)p.uz;
            const double lat2 = rn * rn * (ax * ax + ay * ay + az * az);
            const double sc = 1.0 / sqrt(ca * ca + lat2);
            cos_at = (R)(ca * sc);
            lat = (R)(rn * sc);
        }
        float eps = mc3d_rand_co(&rx, ra);
        refl = eps < Rf;
        tr_ux = refl ? p.ux * ((p.i == nexti) ? 1 : -1)
                     : ((p.i != nexti) ? M::copysign(cos_at, p.ux * cos_at) : p.ux * lat);
        tr_uy = refl ? p.uy * ((p.j == nextj) ? 1 : -1)
                     : (((p.j != nextj) && (p.i == nexti)) ? M::copysign(cos_at, p.uy * cos_at)
                                                           : p.uy * lat);
        tr_uz = refl ? p.uz * ((p.k == nextk) ? 1 : -1)
                     : (((p.k != nextk) && (p.j == nextj) && (p.i == nexti))
                            ? M::copysign(cos_at, p.uz * cos_at)
                            : p.uz * lat);
        (*fresnel_count)++;
    }

    /* absorption, src/mc3d_gpu.cu:262-263 */
    R W = p.W;
    R dW = (mu_t > 0) ? M::albedo_c(tt) * W : 0;
    R W_before = W;
    W = W - dW * (R)(!hit);
    if (AMAP && !hit && mu_t > 0) {
        /* absorption map, the reference's disabled tally (src/mc3d_gpu.cu:265-272):
         * the current voxel clamped into the grid, fixed-point weight removed.  A
         * merged step can end its flight several voxels from where it started, so
         * there the voxel of the interaction point is used. */
        int ai = min(max(JUMP ? nexti : p.i, 0), g.nx - 1);
        int aj = min(max(JUMP ? nextj : p.j, 0), g.ny - 1);
        int ak = min(max(JUMP ? nextk : p.k, 0), g.nz - 1);
        uint64_t dq = M::qw(W_before) - M::qw(W);
        if (dq) atomicAdd(amap + ((int64_t)ak * g.ny + aj) * g.nx + ai, (unsigned long long)dq);
    }

    /* russian roulette, src/mc3d_gpu.cu:275-277 */
    float eps = mc3d_rand_co(&rx, ra);
    bool roulette = M::w_below_threshold(W) && (!hit) && (mu_t != 0);
    if (roulette) {
        R newW = (eps < MC3D_SURVIVAL_LT_F) ? M::roulette_survivor(W) : (R)0;
        /* absorbed weight is booked at the photon's end as Q(W0) - Q(W_end) - lost;
         * a roulette event moves its share from there to the roulette tallies */
        if (newW == 0) {
            uint64_t k = M::qw(W);
            acc[T_RR_KILLED] += k;
            acc[T_ABSORBED] -= k;
        } else {
            uint64_t c = M::qw(newW) - M::qw(W);
            acc[T_RR_CREATED] += c;
            acc[T_ABSORBED] += c;
        }
        W = newW;
    }

    /* Henyey-Greenstein, src/mc3d_gpu.cu:282-294 */
    R costheta = M::template hg_cos<M>(tt, (R)mc3d_rand_oc(&rx, ra));
    R sintheta = M::sqrt(1 - costheta * costheta);
    R phi_divpi = 2 * (R)mc3d_rand_co(&rx, ra);
    R cosphi, sinphi;
    M::sincospi(phi_divpi, &sinphi, &cosphi);
    R invsqrt = M::rsqrt(1 - p.uz * p.uz);
    bool steep = !M::uz_within(M::fabs(p.uz));
    R sc_ux = !steep ? sintheta * (p.ux * p.uz * cosphi - p.uy * sinphi) * invsqrt +
                           p.ux * costheta
                     : sintheta * cosphi;
    R sc_uy = !steep ? sintheta * (p.uy * p.uz * cosphi + p.ux * sinphi) * invsqrt +
                           p.uy * costheta
                     : sintheta * sinphi;
    R sc_uz = !steep ? -1 * M::sqrt(1 - p.uz * p.uz) * sintheta * cosphi + p.uz * costheta
                     : M::copysign(costheta, costheta * p.uz);

    R nux = (!hit) ? sc_ux : tr_ux;
    R nuy = (!hit) ? sc_uy : tr_uy;
    R nuz = (!hit) ? sc_uz : tr_uz;
    const R zero_thresh = M::zero_threshold();
    nux = (M::fabs(nux) < zero_thresh) ? 0 : nux;
    nuy = (M::fabs(nuy) < zero_thresh) ? 0 : nuy;
    nuz = (M::fabs(nuz) < zero_thresh) ? 0 : nuz;
    R norm = M::rsqrt(nux * nux + nuy * nuy + nuz * nuz);
    nux *= norm;
    nuy *= norm;
    nuz *= norm;

    bool freeze = (W <= 0) || (mu_t == 0);
    p.ux = !freeze ? nux : p.ux;
    p.uy = !freeze ? nuy : p.uy;
    p.uz = !freeze ? nuz : p.uz;

    float e2 = mc3d_rand_oc(&rx, ra);
    R newS = (W > 0) ? -M::log((R)e2) : 0;
    p.s = (freeze || hit) ? s : newS;
    p.W = W;

    p.x = !freeze ? newx : p.x;
    p.y = !freeze ? newy : p.y;
    p.z = !freeze ? newz : p.z;

    /* mirror boundary conditions, short-circuited as in src/mc3d_gpu.cu:330; off the
     * lateral faces both mirrors are no-ops, which one rarely taken branch tests */
    bool fres_refl = refl;
    if (!(p.x > 0 && p.x < g.Lx && p.y > 0 && p.y < g.Ly))
        refl = refl || mirror<M>(&p.x, &p.ux, g.Lx) || mirror<M>(&p.y, &p.uy, g.Ly);
    *lat_mirror = refl && !fres_refl;

    bool keep = (hit && refl) || freeze;
    p.i = keep ? p.i : nexti;
    p.j = keep ? p.j : nextj;
    p.k = keep ? p.k : nextk;
    p.tissue = keep ? p.tissue : next_tissue;
    *db_out = db;
    return freeze;
}

/* i, j, k and tissue from the position, as at the start of every launch of
 * photontrack_step (src/mc3d_gpu.cu:168-171). */
template <class M, bool JUMP = false, class R = typename M::real>
static __device__ __forceinline__ void derive_cell(const GeomDev &g, PhotonT<R> &p)
{
    p.i = grid_coord<M>(p.x, p.ux, g.dx, g.rdx);
    p.j = grid_coord<M>(p.y, p.uy, g.dy, g.rdy);
    p.k = grid_coord<M>(p.z, p.uz, g.dz, g.rdz);
    p.tissue = tissue_at<JUMP>(g, p.i, p.j, p.k, p.z, p.uz);
}

/* Whether photontrack_get_grid_coord's face rule puts (x, u) in the stored cell on
 * every axis: strictly inside, or on the lower face moving up, or on the upper face
 * moving down.  Then re-deriving the cell and tissue at a launch boundary changes
 * nothing (above the surface the air rule would apply, which needs z > 0 here). */
template <class R>
static __device__ __forceinline__ bool cell_consistent(const GeomDev &g, const PhotonT<R> &p)
{
    const R xl = (R)p.i * (R)g.dx, xh = (R)(p.i + 1) * (R)g.dx;
    const R yl = (R)p.j * (R)g.dy, yh = (R)(p.j + 1) * (R)g.dy;
    const R zl = (R)p.k * (R)g.dz, zh = (R)(p.k + 1) * (R)g.dz;
    const bool ox = (p.x > xl && p.x < xh) || (p.x == xl && p.ux >= 0) || (p.x == xh && p.ux < 0);
    const bool oy = (p.y > yl && p.y < yh) || (p.y == yl && p.uy >= 0) || (p.y == yh && p.uy < 0);
    const bool oz = (p.z > zl && p.z < zh) || (p.z == zl && p.uz >= 0) || (p.z == zh && p.uz < 0);
    return ox && oy && oz && p.z > 0;
}

template <class R>
static __device__ __forceinline__ bool finite_state(const PhotonT<R> &p)
{
    return isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(p.s) &&
           isfinite(p.ux) && isfinite(p.uy) && isfinite(p.uz);
}

/* The boundary distance the reference's one-voxel DDA (src/mc3d_gpu.cu:29-49,
 * :194) gives a step that starts in state p.  It is 0 when the photon sits on a
 * face of its voxel and moves out through it, which happens when a scattering
 * move rounds onto a voxel face and the new direction points back across it. */
template <class M, class R = typename M::real>
static __device__ __forceinline__ R voxel_db(const GeomDev &g, const PhotonT<R> &p)
{
    R x = p.x, y = p.y, z = p.z;
    return intersection<M>(g, p.i, p.j, p.k, &x, p.ux, &y, p.uy, &z, p.uz);
}

/* The NaN/Inf/db==0 quickfix run after each 45-step launch (src/mc3d_gpu.cu:343-353);
 * zero_db tells whether the launch's last step had db == 0.  Returns true (and
 * zeroes the photon) when it fires. */
template <class R>
static __device__ __forceinline__ bool quickfix(PhotonT<R> &p, bool zero_db)
{
    if (!finite_state(p) || zero_db) {
        p.x = 0; p.y = 0; p.z = 0;
        p.ux = 0; p.uy = 0; p.uz = 1;
        p.W = 0; p.s = 0;
        return true;
    }
    return false;
}

/* The steps a frozen slot keeps executing until the end of its 45-step launch.
 * They change nothing but the mirror (which flips u while the photon sits on a
 * lateral face) and the boundary distance the quickfix looks at. */
template <class M, class R = typename M::real>
static __device__ __forceinline__ R masked_steps(const GeomDev &g, PhotonT<R> &p, int masked, R db)
{
    for (int t = 0; t < masked; t++) {
        R nx_ = p.x, ny_ = p.y, nz_ = p.z;
        db = intersection<M>(g, p.i, p.j, p.k, &nx_, p.ux, &ny_, p.uy, &nz_, p.uz);
        if (!mirror<M>(&p.x, &p.ux, g.Lx)) mirror<M>(&p.y, &p.uy, g.Ly);
    }
    return db;
}

/* --------------------------------------------------------------- kernel body */
static __device__ __forceinline__ void acc_clear(const Acc &a)
{
#pragma unroll
    for (int t = 0; t < MC3D_NUM_TOTALS; t++) a[t] = 0;
}

static __device__ __forceinline__ void acc_flush(const Acc &a, unsigned long long *tot)
{
#pragma unroll
    for (int t = 0; t < MC3D_NUM_TOTALS; t++) {
        unsigned long long v = a[t];
        if (v) atomicAdd(tot + t, v);
        a[t] = 0;
    }
}

/* Multiplier of job-local stream `local`: table line 1 + local mod (L - 1).  The
 * remainder by Barrett reduction with magic = floor((2^64 - 1) / (L - 1)): the
 * quotient estimate is at most one short, so one correction gives the remainder
 * (local < 2^63). */
static __device__ __forceinline__ uint32_t stream_multiplier(const KernelParams &P, int64_t local)
{
    const uint64_t d = (uint64_t)(P.num_multipliers - 1);
    const uint64_t q = __umul64hi((uint64_t)local, P.mult_magic);
    uint64_t r = (uint64_t)local - q * d;
    r = (r >= d) ? r - d : r;
    return P.multipliers[1 + r];
}

/* job owning global stream index gs (binary search over the stream prefix) */
static __device__ __forceinline__ int find_job(const JobDev *jobs, int njobs, int64_t gs)
{
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (jobs[mid].stream_base <= gs) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

/* initial packed state of stream `local` of job `jb` (gpumcml_rng/gpumcml_rng.cu:95-114),
 * honouring the seeding attempts that earlier streams of the job rejected */
static __device__ __forceinline__ uint64_t stream_seed(const KernelParams &P, const JobDev &jb,
                                                       int64_t local, uint32_t fora)
{
    int64_t offset = 0;
    int lo = 0, hi = jb.rej_count - 1;
    while (lo <= hi) { /* last listed stream <= local */
        int mid = (lo + hi) >> 1;
        if (P.rejections[jb.rej_offset + mid].stream <= local) {
            offset = P.rejections[jb.rej_offset + mid].cum;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    uint64_t xs = mc3d_seed_jump(&P.seed, jb.seed, (uint64_t)(local + offset));
    return mc3d_seed_attempt(xs, P.seed.begin, fora);
}

/* The persistent photon loop.  JUMP selects merged steps (photon_step) and needs
 * every geometry's safe-distance map. */
template <class M, bool AMAP, bool JUMP = false, bool ONE_GEOM = false>
__device__ __forceinline__ void photon_kernel_body(const KernelParams &P)
{
    using R = typename M::real;
    /* dynamic shared memory: the optical tables, then (several geometries) the
     * geometry descriptors, read from there instead of being held per thread */
    extern __shared__ float4 sh_tab[];
    __shared__ unsigned long long sh_acc[MC3D_NUM_TOTALS * MC3D_MAX_BLOCK];
    for (int t = threadIdx.x; t < P.props_entries; t += blockDim.x) sh_tab[t] = P.props_table[t];
    GeomDev *sh_geom = reinterpret_cast<GeomDev *>(sh_tab + P.props_entries);
    if (!ONE_GEOM)
        for (int t = threadIdx.x; t < P.ngeoms; t += blockDim.x) sh_geom[t] = P.geoms[t];
    const Acc acc{sh_acc + threadIdx.x};
    acc_clear(acc);
    __syncthreads();

    int job = -1;
    const GeomDev *gp = sh_geom;
    const float4 *tab = sh_tab;
    int64_t left = 0, local = 0;
    uint64_t rx = 0;
    uint32_t ra = 1;
    PhotonT<R> p;
    bool alive = false;
    int chunk = 0;
    /* Loop iterations modulo the 45-step chunk.  A photon starts only at tick 0,
     * as a reference slot starts only at a launch boundary: a lane whose photon
     * ended waits out the rest of the chunk (the reference's masked steps), so
     * the lanes of a warp reach their chunk ends on the same iteration. */
    int tick = 0;
    uint32_t psteps = 0;
    uint32_t fresnel = 0;
    unsigned long long *amap = nullptr;

    for (;;) {
        if (!alive) {
            if (tick != 0) {
                tick = (tick == MC3D_NUM_PHOTON_STEPS - 1) ? 0 : tick + 1;
                continue;
            }
            if (left == 0) {
                if (P.cancel && *((volatile const int *)P.cancel)) break;
                int64_t gs = (int64_t)atomicAdd((unsigned long long *)P.work_counter, 1ull);
                if (gs >= P.total_streams) break;
                const int next_job = find_job(P.jobs, P.njobs, gs);
                /* the per-thread tallies are the job's: flushed when the job changes */
                if (job >= 0 && next_job != job)
                    acc_flush(acc, P.totals + (int64_t)job * MC3D_NUM_TOTALS);
                job = next_job;
                const JobDev &jb = P.jobs[job];
                gp = sh_geom + jb.geom;
                tab = sh_tab + jb.props_offset;
                if (AMAP) amap = P.amap + jb.amap_offset;
                local = gs - jb.stream_base + jb.stream_first;
                left = jb.per_stream + (local < jb.remainder ? 1 : 0);
                ra = stream_multiplier(P, local);
                rx = stream_seed(P, jb, local, ra);
                if (left == 0) continue;
            }
            const GeomDev &g = ONE_GEOM ? P.geom0 : *gp;
            /* photontrack_reinitialize, src/mc3d_gpu.cu:74-111 */
            if (P.jobs[job].beam == 0) {
                p.x = (R)g.Lx * (R)mc3d_rand_co(&rx, ra);
                p.y = (R)g.Ly * (R)mc3d_rand_co(&rx, ra);
            } else {
                p.x = (R)g.Lx / 2;
                p.y = (R)g.Ly / 2;
            }
            p.z = 0;
            p.ux = 0; p.uy = 0; p.uz = 1;
            /* specular reflection from air into tissue type 1 (src/mc3d_gpu.cu:67-70, 500) */
            const R n0 = M::n(tab + MC3D_TAB_STRIDE * MC3D_TISSUE_AIR), n1 = M::n(tab + MC3D_TAB_STRIDE);
            R rsp = M::div(n0 - n1, n0 + n1);
            rsp = rsp * rsp;
            p.W = (R)1 - rsp;
            p.s = -M::log((R)mc3d_rand_oc(&rx, ra));
            derive_cell<M, JUMP>(g, p);
            chunk = 0;
            psteps = 0;
            fresnel = 0;
            alive = true;
            left--;
        }

        const GeomDev &g = ONE_GEOM ? P.geom0 : *gp;
        R db;
        bool lat_mirror;
        bool froze;
        /* Merged steps: the quickfix must see the boundary distance of the
         * reference's one-voxel DDA for the chunk's last step, not the merged
         * box's (which is never 0 inside a uniform cube), or merged steps would
         * lose less weight to it than the reference does.  Taken from that
         * step's start state. */
        bool vzero = false;
        if (JUMP && chunk == MC3D_NUM_PHOTON_STEPS - 1) vzero = voxel_db<M>(g, p) == 0;
        froze = photon_step<M, AMAP, JUMP>(g, tab, p, rx, ra, acc, &db, &fresnel, amap,
                                           &lat_mirror);
        chunk++;
        psteps++;
        tick = (tick == MC3D_NUM_PHOTON_STEPS - 1) ? 0 : tick + 1;

        bool done = false;
        uint64_t lost = 0;
        if (froze) {
            /* If the freeze step's mirror did not fire and the photon is off the
             * lateral faces, the masked steps change nothing and see the freeze
             * step's boundary distance again: no need to replay them.  The
             * replayed masked steps are one-voxel steps; without them a merged
             * kernel takes the one-voxel distance of the frozen state, which is
             * the freeze step's start state. */
            bool zero;
            if (lat_mirror || !(p.x > 0 && p.x < g.Lx && p.y > 0 && p.y < g.Ly)) {
                if (chunk < MC3D_NUM_PHOTON_STEPS)
                    zero = masked_steps<M>(g, p, MC3D_NUM_PHOTON_STEPS - chunk, db) == 0;
                else
                    zero = JUMP ? vzero : db == 0;
            } else {
                zero = JUMP ? voxel_db<M>(g, p) == 0 : db == 0;
            }
            R w_before = p.W;
            if (quickfix(p, zero)) { acc[T_QUICKFIX]++; lost = M::qw(w_before); }
            done = true;
        } else if (chunk == MC3D_NUM_PHOTON_STEPS) {
            R w_before = p.W;
            if (quickfix(p, JUMP ? vzero : db == 0)) {
                acc[T_QUICKFIX]++;
                lost = M::qw(w_before);
                done = true;
            } else {
                /* fast math: re-derive only where the stored cell breaks the face rule
                 * (exact math always re-derives, as the reference's relaunch does) */
                if (!M::kFast || !cell_consistent(g, p)) derive_cell<M, JUMP>(g, p);
                chunk = 0;
            }
        }
        if (!done && (int64_t)psteps >= P.max_steps) {
            lost = M::qw(p.W);
            p.W = 0;
            acc[T_CAPPED]++;
            done = true;
        }
        if (done) {
            /* photon_detector, src/mc3d_photons.cu:151-171 */
            const JobDev &jb = P.jobs[job];
            int ix = grid_coord<M>(p.x, p.ux, g.dx, g.rdx);
            int iy = grid_coord<M>(p.y, p.uy, g.dy, g.rdy);
            bool inside = (ix >= 0) && (iy >= 0) && (ix < g.nx) && (iy < g.ny);
            uint64_t q = M::qw(p.W);
            int64_t bin = jb.bin_offset + (int64_t)iy * g.nx + ix;
            int slot;
            if (p.z <= 0) {
                slot = inside ? T_R_IN : T_R_OUT;
                if (inside && q) {
                    atomicAdd(P.drs + bin, (unsigned long long)q);
                    atomicAdd(P.drs_sq + bin, (unsigned long long)M::qw(p.W * p.W));
                }
            } else {
                slot = inside ? T_T_IN : T_T_OUT;
                if (inside && q) atomicAdd(P.trans + bin, (unsigned long long)q);
            }
            acc[slot] += q;
            /* the launch weight 1 - Rsp again, as at the photon's start */
            const R n0 = M::n(tab + MC3D_TAB_STRIDE * MC3D_TISSUE_AIR), n1 = M::n(tab + MC3D_TAB_STRIDE);
            R rsp = M::div(n0 - n1, n0 + n1);
            rsp = rsp * rsp;
            const uint64_t qw0 = M::qw((R)1 - rsp);
            acc[T_W_LAUNCHED] += qw0;
            acc[T_ABSORBED] += qw0 - q - lost;
            acc[T_LOST] += lost;
            acc[T_PHOTONS] += 1;
            acc[T_STEPS] += psteps;
            acc[T_FRESNEL] += fresnel;
            if (P.photon_log) {
                int64_t nstream = jb.per_stream + (local < jb.remainder ? 1 : 0);
                int64_t kphot = nstream - left - 1;
                int64_t pid = jb.photon_base + local + kphot * jb.streams;
                PhotonRecord r;
                r.x = (float)p.x; r.y = (float)p.y; r.z = (float)p.z;
                r.ux = (float)p.ux; r.uy = (float)p.uy; r.uz = (float)p.uz;
                r.W = (float)p.W; r.s = (float)p.s;
                r.steps = psteps;
                r.tissue = (uint32_t)(p.tissue & 0xff);
                r.rng = rx;
                P.photon_log[pid] = r;
            }
            alive = false;
        }
    }
    if (job >= 0) acc_flush(acc, P.totals + (int64_t)job * MC3D_NUM_TOTALS);
}

} /* namespace mc3d */

#endif /* MC3D_ENGINE_CUH */
