/*
 * mc3d_oracle.c -- CPU restatement of YMC3D's photon-tracking path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke test
 * and bench.py's CPU-baseline leg load it; the engine never does.  It restates
 * the reference line by line, in plain C, scalar, FP32:
 *   init_RNG / rand_MWC_co / rand_MWC_oc   gpumcml_rng/gpumcml_rng.cu:38-118
 *   photontrack_get_grid_coord             src/mc3d_gpu.cu:53-63
 *   photontrack_get_tissue_type            src/mc3d_gpu.cu:24-27 (+ clamp addressing :416-418)
 *   photontrack_intersection               src/mc3d_gpu.cu:29-49
 *   photontrack_calc_specular_reflection   src/mc3d_gpu.cu:67-70
 *   photontrack_reinitialize               src/mc3d_gpu.cu:74-111 (both beam branches,
 *                                          the pencil one without its shadowing bug)
 *   photontrack_mirror                     src/mc3d_gpu.cu:113-126
 *   photontrack_step                       src/mc3d_gpu.cu:128-376
 *   photon_detector                        src/mc3d_photons.cu:151-171
 * with the slot structure of run_3dmc_gpu (src/mc3d_gpu.cu:483-584) expressed per
 * photon: a slot starts every photon at a 45-step launch boundary, re-derives
 * i,j,k every 45 steps, applies the NaN/db==0 quickfix at the end of each launch,
 * and keeps stepping (masked) after a freeze until the launch ends.  A stream
 * (slot) runs its photons one after another on one generator; the masked steps'
 * random draws of the reference are not made (they are discarded there).
 *
 * Elementary functions come from ymc3d_b200/csrc/mc3d_exactmath.h so that, built
 * with -ffp-contract=off, every operation matches the engine's exact-math kernel
 * bit for bit.  Tallies use the engine's fixed point, Q(W) = round(W 2^32).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../ymc3d_b200/csrc/mc3d_exactmath.h"

/* The transport arithmetic type.  The default build is FP32, like the reference,
 * with the reproducible series functions; -DORC_F64 builds the same loop in FP64
 * with libm's functions, the precision reference for FP32 results. */
#ifdef ORC_F64
typedef double real;
#define R_FMIN fmin
#define R_FLOOR floor
#define R_FABS fabs
#define R_COPYSIGN copysign
#define R_SQRT sqrt
#define R_LOG log
#define R_ACOS acos
#define R_SIN sin
static void r_sincospi(double x, double *s, double *c)
{
    *s = sin(3.14159265358979323846 * x);
    *c = cos(3.14159265358979323846 * x);
}
#else
typedef float real;
#define R_FMIN fminf
#define R_FLOOR floorf
#define R_FABS fabsf
#define R_COPYSIGN copysignf
#define R_SQRT sqrtf
#define R_LOG mc3d_xm_logf
#define R_ACOS mc3d_xm_acosf
#define R_SIN mc3d_xm_sinf
#define r_sincospi mc3d_xm_sincospif
#endif

#define ORC_SURVIVAL_CHANCE 0.1 /* src/mc3d_types.h:11-18 */
#define ORC_W_THRESHOLD 0.0001
#define ORC_UZ_THRESH 0.99999
#define ORC_NUM_PHOTON_STEPS 45
#define ORC_AIR 0
#define ORC_NTOT 14

typedef struct {
    int32_t nx, ny, nz, pad;
    double dx, dy, dz; /* file values; used as float like geometry_t */
    const uint8_t *tissue;
} orc_geom;

typedef struct {
    int32_t ntypes, pad;
    const float *mua, *mus, *g, *n;
} orc_props;

typedef struct {
    int64_t photons, streams; /* streams must be > 0 */
    uint64_t seed;
    int32_t beam, pad;
    int64_t max_steps;
} orc_job;

typedef struct {
    float x, y, z, ux, uy, uz, W, s;
    uint32_t steps, tissue;
    uint64_t rng;
} orc_rec;

/* ------------------------------------------------------------------ RNG */

static float orc_u32_to_float_rz(uint32_t u)
{
    if (u < (1u << 24)) return (float)u;
    int drop = 8 - __builtin_clz(u);
    return (float)(u & ~((1u << drop) - 1u));
}

static float orc_rand_co1(uint64_t *x, uint32_t a)
{
    *x = (*x & 0xffffffffull) * a + (*x >> 32);
    return orc_u32_to_float_rz((uint32_t)*x) * 0x1p-32f;
}

static float orc_rand_oc1(uint64_t *x, uint32_t a) { return 1.0f - orc_rand_co1(x, a); }

void orc_rand_co(uint64_t *x, uint32_t a, int64_t n, float *out)
{
    for (int64_t i = 0; i < n; i++) out[i] = orc_rand_co1(x, a);
}

/* init_RNG, one stream after another.  Streams beyond the table reuse its
 * multipliers cyclically (the reference's fscanf would repeat the last one). */
int orc_init_rng(const uint32_t *table, int64_t table_len, uint64_t xinit, int64_t n,
                 uint64_t *x, uint32_t *a)
{
    if (table_len < 2) return 3;
    uint32_t begin = table[0];
    if ((xinit == 0ull) | (((uint32_t)(xinit >> 32)) >= (begin - 1u)) |
        (((uint32_t)xinit) >= 0xffffffffu))
        return 1;
    for (int64_t i = 0; i < n; i++) {
        uint32_t fora = table[1 + i % (table_len - 1)];
        uint64_t st = 0;
        int tries = 0;
        while ((st == 0ull) | (((uint32_t)(st >> 32)) >= (fora - 1u)) |
               (((uint32_t)st) >= 0xffffffffu)) {
            if (++tries > 4096) return 2;
            xinit = (xinit & 0xffffffffull) * begin + (xinit >> 32);
            st = (uint32_t)floor((((double)((uint32_t)xinit)) / (double)0x100000000ull) * fora);
            st = st << 32;
            xinit = (xinit & 0xffffffffull) * begin + (xinit >> 32);
            st += (uint32_t)xinit;
        }
        x[i] = st;
        a[i] = fora;
    }
    return 0;
}

/* --------------------------------------------------------------- helpers */

/* real -> int as the GPU converts (saturating, NaN -> 0) */
static int orc_f2i(real v)
{
    if (v != v) return 0;
    if (v >= (real)2147483648.0) return INT32_MAX;
    if (v < (real)-2147483648.0) return INT32_MIN;
    return (int)v;
}

static int orc_inc(int i) { return (int)((unsigned)i + 1u); }

static int orc_grid_coord(real x, real ux, real d)
{
    int i = orc_f2i(R_FLOOR(x / d));
    i += (x == (real)orc_inc(i) * d);
    real bmin = (real)i * d;
    i = ((x > bmin) || ((x == bmin) && (ux >= 0))) ? i : i - 1;
    return i;
}

typedef struct {
    int nx, ny, nz;
    real dx, dy, dz, Lx, Ly, Lz;
    const uint8_t *tissue;
} orc_g;

static int orc_clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int orc_tissue(const orc_g *g, int i, int j, int k, real z, real uz)
{
    int ci = orc_clampi(i, 0, g->nx - 1);
    int cj = orc_clampi(j, 0, g->ny - 1);
    int ck = orc_clampi(k, 0, g->nz - 1);
    int t = g->tissue[((int64_t)ck * g->ny + cj) * g->nx + ci];
    return ((z <= 0) && (uz < 0)) ? ORC_AIR : t;
}

static real orc_intersection(const orc_g *g, int i, int j, int k, real *x, real ux, real *y,
                              real uy, real *z, real uz)
{
    real border_x = (real)((ux >= 0) ? orc_inc(i) : i) * g->dx;
    real t_x = (border_x - *x) / ux;
    real border_y = (real)((uy >= 0) ? orc_inc(j) : j) * g->dy;
    real t_y = (border_y - *y) / uy;
    real border_z = (real)((uz >= 0) ? orc_inc(k) : k) * g->dz;
    real t_z = (border_z - *z) / uz;
    real t = R_FMIN(t_x, R_FMIN(t_y, t_z));
    *x = (t == t_x) ? border_x : *x + ux * t;
    *y = (t == t_y) ? border_y : *y + uy * t;
    *z = (t == t_z) ? border_z : *z + uz * t;
    return t;
}

static int orc_mirror(real *x, real *ux, real length)
{
    int refl = (*x >= length) || (*x <= 0);
    *x = (*x >= length) ? 2 * length - *x : *x;
    *x = (*x <= 0) ? R_FABS(*x) : *x;
    *ux = refl ? -1 * (*ux) : *ux;
    return refl;
}

static uint64_t orc_q(real w)
{
    double v = nearbyint((double)(w * (real)4294967296.0));
    if (!(v > 0)) return 0; /* negative and NaN convert to 0, as cvt.rni.u64 does */
    if (v >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)v;
}

typedef struct {
    real x, y, z, ux, uy, uz, W, s;
    int i, j, k, tissue;
} orc_ph;

typedef struct {
    const real *mua, *mus, *g, *n;
} orc_tab;

/* photontrack_step body for one live photon; returns 1 on freeze */
static int orc_step(const orc_g *G, const orc_tab *P, orc_ph *p, uint64_t *rx, uint32_t ra,
                    uint64_t *killed, uint64_t *created, real *db_out, uint64_t *fresnel,
                    uint64_t *amap)
{
    int tissue_type = p->tissue;
    real ni = P->n[tissue_type];
    real nt = ni;
    real epsilon;
    real mu_a = P->mua[tissue_type];
    real mu_s = P->mus[tissue_type];
    real g = P->g[tissue_type];
    real mu_t = mu_a + mu_s;

    real newx = p->x, newy = p->y, newz = p->z;
    real db = orc_intersection(G, p->i, p->j, p->k, &newx, p->ux, &newy, p->uy, &newz, p->uz);

    int hit_boundary = db * mu_t <= p->s;
    real ds = hit_boundary ? db * mu_t : p->s;
    newx = hit_boundary ? newx : p->x + p->ux * ds / mu_t;
    newy = hit_boundary ? newy : p->y + p->uy * ds / mu_t;
    newz = hit_boundary ? newz : p->z + p->uz * ds / mu_t;
    real s = p->s - ds;

    int nexti = orc_grid_coord(newx, p->ux, G->dx);
    int nextj = orc_grid_coord(newy, p->uy, G->dy);
    int nextk = orc_grid_coord(newz, p->uz, G->dz);
    int next_tissue_type = orc_tissue(G, nexti, nextj, nextk, newz, p->uz);
    nt = P->n[next_tissue_type];

    real ux = p->ux, uy = p->uy, uz = p->uz;
    real transrefl_ux = ux, transrefl_uy = uy, transrefl_uz = uz;
    int isReflected = 0;
    if (ni != nt) {
        real cos_ai = (p->i != nexti) ? ux : ((p->j != nextj) ? uy : uz);
        cos_ai = R_FABS(cos_ai);
        cos_ai = (cos_ai > 1) ? 1 : cos_ai;
        real ai = R_ACOS(cos_ai);
        real ni_nt = ni / nt;
        real sin_ai = R_SIN(ai);
        real sin_at = ni_nt * sin_ai;
        real cos_at = R_SQRT((real)1 - sin_at * sin_at);
        real R1 = (sin_ai * cos_at - cos_ai * sin_at) / (sin_ai * cos_at + cos_ai * sin_at);
        real R2 = (cos_ai * cos_at - sin_ai * sin_at) / (cos_ai * cos_at + sin_at * sin_at);
        real R = 0.5 * R1 * R1 * ((real)1 + R2 * R2);
        R = (sin_at > 1) ? 1 : R;
        R = (ni == nt) ? 0 : R;
        epsilon = orc_rand_co1(rx, ra);
        isReflected = epsilon < R;
        transrefl_ux = isReflected ? ux * ((p->i == nexti) ? 1 : -1)
                                   : ((p->i != nexti) ? R_COPYSIGN(cos_at, ux * cos_at) : ux * ni_nt);
        transrefl_uy = isReflected ? uy * ((p->j == nextj) ? 1 : -1)
                                   : (((p->j != nextj) && (p->i == nexti))
                                          ? R_COPYSIGN(cos_at, uy * cos_at)
                                          : uy * ni_nt);
        transrefl_uz = isReflected ? uz * ((p->k == nextk) ? 1 : -1)
                                   : (((p->k != nextk) && (p->j == nextj) && (p->i == nexti))
                                          ? R_COPYSIGN(cos_at, uz * cos_at)
                                          : uz * ni_nt);
        (*fresnel)++;
    }

    real W = p->W;
    real dW = (mu_t > 0) ? mu_a / mu_t * W : 0;
    W = W - dW * (real)(!hit_boundary);
    if (amap && (!hit_boundary) && (mu_t > 0)) {
        /* the reference's disabled absorption tally (src/mc3d_gpu.cu:265-272) */
        int abs_i = orc_clampi(p->i, 0, G->nx - 1);
        int abs_j = orc_clampi(p->j, 0, G->ny - 1);
        int abs_k = orc_clampi(p->k, 0, G->nz - 1);
        uint64_t dq = orc_q(p->W) - orc_q(W);
#pragma omp atomic
        amap[((int64_t)abs_k * G->ny + abs_j) * G->nx + abs_i] += dq;
    }

    epsilon = orc_rand_co1(rx, ra);
    real newW = (epsilon < ORC_SURVIVAL_CHANCE) ? (real)(W / ORC_SURVIVAL_CHANCE) : 0;
    if ((W < ORC_W_THRESHOLD) && (!hit_boundary) && (mu_t != 0)) {
        if (newW == 0.0f) *killed += orc_q(W);
        else *created += orc_q(newW) - orc_q(W);
        W = newW;
    }

    real costheta = (1 - g * g) / (1 - g + 2 * g * orc_rand_oc1(rx, ra));
    costheta = (real)1 / (2 * g) * (1 + g * g - costheta * costheta);
    real sintheta = R_SQRT(1 - costheta * costheta);
    real phi_divpi = 2 * orc_rand_co1(rx, ra);
    real cosphi, sinphi;
    r_sincospi(phi_divpi, &sinphi, &cosphi);
    real invsqrt = (real)1 / R_SQRT(1 - uz * uz);
    real scatt_ux = (R_FABS(uz) <= ORC_UZ_THRESH)
                         ? sintheta * (ux * uz * cosphi - uy * sinphi) * invsqrt + ux * costheta
                         : sintheta * cosphi;
    real scatt_uy = (R_FABS(uz) <= ORC_UZ_THRESH)
                         ? sintheta * (uy * uz * cosphi + ux * sinphi) * invsqrt + uy * costheta
                         : sintheta * sinphi;
    real scatt_uz = (R_FABS(uz) <= ORC_UZ_THRESH)
                         ? -1 * R_SQRT(1 - uz * uz) * sintheta * cosphi + uz * costheta
                         : R_COPYSIGN(costheta, costheta * uz);

    real newux = (!hit_boundary) ? scatt_ux : transrefl_ux;
    real newuy = (!hit_boundary) ? scatt_uy : transrefl_uy;
    real newuz = (!hit_boundary) ? scatt_uz : transrefl_uz;
    real zero_thresh = 1 - ORC_UZ_THRESH;
    newux = (R_FABS(newux) < zero_thresh) ? 0 : newux;
    newuy = (R_FABS(newuy) < zero_thresh) ? 0 : newuy;
    newuz = (R_FABS(newuz) < zero_thresh) ? 0 : newuz;
    real newu_norm = (real)1 / R_SQRT(newux * newux + newuy * newuy + newuz * newuz);
    newux *= newu_norm;
    newuy *= newu_norm;
    newuz *= newu_norm;

    int freeze = (W <= 0) || (mu_t == 0);
    p->ux = (!freeze) ? newux : ux;
    p->uy = (!freeze) ? newuy : uy;
    p->uz = (!freeze) ? newuz : uz;

    epsilon = orc_rand_oc1(rx, ra);
    real newS = (W > 0) ? -R_LOG(epsilon) : 0;
    p->s = (freeze || hit_boundary) ? s : newS;
    p->W = W;

    p->x = (!freeze) ? newx : p->x;
    p->y = (!freeze) ? newy : p->y;
    p->z = (!freeze) ? newz : p->z;

    isReflected = isReflected || orc_mirror(&p->x, &p->ux, G->Lx) || orc_mirror(&p->y, &p->uy, G->Ly);

    int keep = (hit_boundary && isReflected) || freeze;
    p->i = keep ? p->i : nexti;
    p->j = keep ? p->j : nextj;
    p->k = keep ? p->k : nextk;
    p->tissue = keep ? p->tissue : next_tissue_type;
    *db_out = db;
    return freeze;
}

static void orc_derive(const orc_g *G, orc_ph *p)
{
    p->i = orc_grid_coord(p->x, p->ux, G->dx);
    p->j = orc_grid_coord(p->y, p->uy, G->dy);
    p->k = orc_grid_coord(p->z, p->uz, G->dz);
    p->tissue = orc_tissue(G, p->i, p->j, p->k, p->z, p->uz);
}

static int orc_quickfix(orc_ph *p, real db)
{
    if (isinf(p->x) || isnan(p->x) || isinf(p->y) || isnan(p->y) || isinf(p->z) || isnan(p->z) ||
        isinf(p->s) || isnan(p->s) || isinf(p->ux) || isnan(p->ux) || isinf(p->uy) ||
        isnan(p->uy) || isinf(p->uz) || isnan(p->uz) || (db == 0)) {
        p->x = 0; p->y = 0; p->z = 0;
        p->ux = 0; p->uy = 0; p->uz = 1;
        p->W = 0; p->s = 0;
        return 1;
    }
    return 0;
}

typedef struct {
    uint64_t t[ORC_NTOT];
    uint64_t *drs, *drs_sq, *trans;
} orc_acc;

/* one photon of a slot, from reinitialisation to the detector */
static void orc_photon(const orc_g *G, const orc_tab *P, int beam, int64_t max_steps, uint64_t *rx,
                       uint32_t ra, orc_acc *acc, orc_rec *rec, uint64_t *amap)
{
    orc_ph p;
    if (beam == 0) {
        p.x = G->Lx * orc_rand_co1(rx, ra);
        p.y = G->Ly * orc_rand_co1(rx, ra);
    } else {
        p.x = G->Lx / 2;
        p.y = G->Ly / 2;
    }
    p.z = 0;
    p.ux = 0; p.uy = 0; p.uz = 1;
    real n0 = P->n[ORC_AIR], n1 = P->n[1];
    real Rsp = (n0 - n1) / (n0 + n1);
    Rsp = Rsp * Rsp;
    p.W = (real)1 - Rsp;
    p.s = -R_LOG(orc_rand_oc1(rx, ra));
    uint64_t q0 = orc_q(p.W);
    orc_derive(G, &p);

    uint64_t killed = 0, created = 0, lost = 0, fresnel = 0;
    int chunk = 0;
    int64_t steps = 0;
    for (;;) {
        real db;
        int froze = orc_step(G, P, &p, rx, ra, &killed, &created, &db, &fresnel, amap);
        chunk++;
        steps++;
        int done = 0;
        if (froze) {
            /* the rest of the 45-step launch: masked steps (mirror + boundary distance) */
            for (int m = chunk; m < ORC_NUM_PHOTON_STEPS; m++) {
                real nx_ = p.x, ny_ = p.y, nz_ = p.z;
                db = orc_intersection(G, p.i, p.j, p.k, &nx_, p.ux, &ny_, p.uy, &nz_, p.uz);
                if (!orc_mirror(&p.x, &p.ux, G->Lx)) orc_mirror(&p.y, &p.uy, G->Ly);
            }
            real wb = p.W;
            if (orc_quickfix(&p, db)) { acc->t[12]++; lost = orc_q(wb); }
            done = 1;
        } else if (chunk == ORC_NUM_PHOTON_STEPS) {
            real wb = p.W;
            if (orc_quickfix(&p, db)) { acc->t[12]++; lost = orc_q(wb); done = 1; }
            else { orc_derive(G, &p); chunk = 0; }
        }
        if (!done && steps >= max_steps) {
            lost = orc_q(p.W);
            p.W = 0;
            acc->t[11]++;
            done = 1;
        }
        if (done) break;
    }
    /* photon_detector */
    int ind_x = orc_grid_coord(p.x, p.ux, G->dx);
    int ind_y = orc_grid_coord(p.y, p.uy, G->dy);
    int inside = (ind_x >= 0) && (ind_y >= 0) && (ind_x < G->nx) && (ind_y < G->ny);
    uint64_t q = orc_q(p.W);
    int64_t bin = (int64_t)ind_y * G->nx + ind_x;
    if (p.z <= 0) {
        if (inside) {
            acc->drs[bin] += q;
            acc->drs_sq[bin] += orc_q(p.W * p.W);
            acc->t[3] += q;
        } else {
            acc->t[4] += q;
        }
    } else {
        if (inside) {
            acc->trans[bin] += q;
            acc->t[5] += q;
        } else {
            acc->t[6] += q;
        }
    }
    acc->t[0]++;
    acc->t[1] += (uint64_t)steps;
    acc->t[2] += q0;
    acc->t[7] += q0 - q - killed + created - lost;
    acc->t[8] += killed;
    acc->t[9] += created;
    acc->t[10] += lost;
    acc->t[13] += fresnel;
    if (rec) {
        rec->x = p.x; rec->y = p.y; rec->z = p.z;
        rec->ux = p.ux; rec->uy = p.uy; rec->uz = p.uz;
        rec->W = p.W; rec->s = p.s;
        rec->steps = (uint32_t)steps;
        rec->tissue = (uint32_t)p.tissue;
        rec->rng = *rx;
    }
}

/* Simulate streams [first, first + count) of a job (count < 0: to the end).
 * Bin arrays are nx*ny and accumulated into; totals[14] likewise (order of
 * mc3d_totals).  log, if given, has one record per photon of the whole job; amap, if
 * given, is nz*ny*nx and accumulates the absorbed fixed-point weight per voxel. */
int orc_run(const orc_geom *geom, const orc_props *props, const orc_job *job,
            const uint32_t *table, int64_t table_len, int nthreads, int64_t first, int64_t count,
            uint64_t *drs, uint64_t *drs_sq, uint64_t *trans, uint64_t *totals, orc_rec *log,
            uint64_t *amap)
{
    if (job->streams <= 0 || props->ntypes < 2) return 4;
    int64_t S = job->streams;
    if (count < 0 || first + count > S) count = S - first;
    if (first < 0 || count < 0) return 4;
    int64_t nseed = first + count;
    uint64_t *sx = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(nseed ? nseed : 1));
    uint32_t *sa = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nseed ? nseed : 1));
    int st = orc_init_rng(table, table_len, job->seed, nseed, sx, sa);
    if (st) {
        free(sx);
        free(sa);
        return st;
    }
    orc_g G;
    G.nx = geom->nx; G.ny = geom->ny; G.nz = geom->nz;
    G.dx = (real)geom->dx; G.dy = (real)geom->dy; G.dz = (real)geom->dz;
    G.Lx = G.dx * G.nx; G.Ly = G.dy * G.ny; G.Lz = G.dz * G.nz;
    G.tissue = geom->tissue;
    /* optical properties in the transport type (the file values are float) */
    real *tabv = (real *)malloc(sizeof(real) * 4 * (size_t)props->ntypes);
    for (int t = 0; t < props->ntypes; t++) {
        tabv[t] = props->mua[t];
        tabv[props->ntypes + t] = props->mus[t];
        tabv[2 * props->ntypes + t] = props->g[t];
        tabv[3 * props->ntypes + t] = props->n[t];
    }
    orc_tab P = {tabv, tabv + props->ntypes, tabv + 2 * props->ntypes, tabv + 3 * props->ntypes};
    int64_t nb = (int64_t)G.nx * G.ny;
    int64_t per = job->photons / S, rem = job->photons % S;
    int64_t max_steps = job->max_steps > 0 ? job->max_steps : (1 << 24);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel
    {
        orc_acc acc;
        memset(acc.t, 0, sizeof acc.t);
        acc.drs = (uint64_t *)calloc((size_t)nb, sizeof(uint64_t));
        acc.drs_sq = (uint64_t *)calloc((size_t)nb, sizeof(uint64_t));
        acc.trans = (uint64_t *)calloc((size_t)nb, sizeof(uint64_t));
#pragma omp for schedule(dynamic, 16)
        for (int64_t i = first; i < first + count; i++) {
            uint64_t rx = sx[i];
            uint32_t ra = sa[i];
            int64_t np = per + (i < rem ? 1 : 0);
            for (int64_t k = 0; k < np; k++) {
                orc_rec *rec = log ? &log[i + k * S] : NULL;
                orc_photon(&G, &P, job->beam, max_steps, &rx, ra, &acc, rec, amap);
            }
        }
#pragma omp critical
        {
            for (int64_t b = 0; b < nb; b++) {
                drs[b] += acc.drs[b];
                drs_sq[b] += acc.drs_sq[b];
                trans[b] += acc.trans[b];
            }
            for (int t = 0; t < ORC_NTOT; t++) totals[t] += acc.t[t];
        }
        free(acc.drs);
        free(acc.drs_sq);
        free(acc.trans);
    }
    free(sx);
    free(sa);
    free(tabv);
    return 0;
}

/* exact-math primitives, exported for the accuracy tests */
float orc_logf(float x) { return mc3d_xm_logf(x); }
float orc_acosf(float x) { return mc3d_xm_acosf(x); }
float orc_sinf(float x) { return mc3d_xm_sinf(x); }
void orc_sincospif(float x, float *s, float *c) { mc3d_xm_sincospif(x, s, c); }
int orc_grid_coord_x(float x, float ux, float d) { return orc_grid_coord(x, ux, d); }
