/*
 * mc3d.h -- C ABI of the B200 photon-tracking engine (libmc3d.so).
 *
 * Replaces the GPU path of YMC3D: the host driver
 *     void run_3dmc_gpu(geometry_t, opticalprops_t, int num_photons, double *R,
 *                       double *R_tot, double *T, double *T_tot, float *A,
 *                       int *num_finished_photons)        (src/mc3d_gpu.h:16,
 *                                                           src/mc3d_gpu.cu:388-601)
 * with its kernels photontrack_reinitialize / photontrack_step
 * (src/mc3d_gpu.cu:74-376), the host reflectance detector photon_detector
 * (src/mc3d_photons.cu:151-171) and the RNG seeding rng_init / init_RNG
 * (src/mc3d_rng.cu:12-37, gpumcml_rng/gpumcml_rng.cu:59-118); plus the file
 * formats of src/mc3d_io.cu:16-255.
 *
 * Conventions: plain pointers and sizes, caller-owned host buffers, every call
 * returns a status (0 = MC3D_OK, negative = error; mc3d_last_error() gives text).
 * Weights are tallied in unsigned 64-bit fixed point, Q(W) = round(W * 2^32), so
 * sums are exact and independent of execution order.
 */
#ifndef MC3D_H
#define MC3D_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC3D_ABI_VERSION 2
#define MC3D_WEIGHT_SCALE 4294967296.0 /* 2^32: fixed-point units per unit weight */

enum mc3d_status {
    MC3D_OK = 0,
    MC3D_ERR_ARG = -1,          /* null pointer, bad count or index */
    MC3D_ERR_GEOMETRY = -2,     /* non-positive size or voxel size */
    MC3D_ERR_TISSUE_RANGE = -3, /* a voxel names a tissue type the optical set lacks */
    MC3D_ERR_PROPS = -4,        /* fewer than 2 tissue types (air + one) or a bad value */
    MC3D_ERR_SEED = -5,         /* seed invalid for the table's seeding multiplier */
    MC3D_ERR_TABLE = -6,        /* safe-prime table missing or shorter than 2 lines */
    MC3D_ERR_CUDA = -7,         /* CUDA runtime error (text in mc3d_last_error) */
    MC3D_ERR_NO_DEVICE = -8,
    MC3D_ERR_IO = -9,           /* file cannot be opened / written */
    MC3D_ERR_FORMAT = -10,      /* malformed or truncated file */
    MC3D_ERR_CAPACITY = -11,    /* optical tables of one launch exceed shared memory */
    MC3D_ERR_CANCELLED = -12    /* the cancel flag stopped the run; results are partial */
};

enum mc3d_beam { MC3D_BEAM_UNIFORM = 0, MC3D_BEAM_PENCIL = 1 };
/* FAST: FP32 with the GPU's approximate division, sqrt, log and sin, as the
 * reference's -use_fast_math build.  EXACT: FP32 with IEEE operations and
 * reproducible series functions, bit-identical to the CPU transcription.  F64:
 * the same loop stepping in FP64, the precision reference (no counterpart in the
 * reference). */
enum mc3d_math { MC3D_MATH_FAST = 0, MC3D_MATH_EXACT = 1, MC3D_MATH_F64 = 2 };

/* Step decomposition of the fast-math kernel.  MERGED (the default) runs each
 * step's voxel traversal on the cube of voxels around the photon's voxel that
 * holds only its tissue (a per-voxel safe-distance map, built when the plan is
 * created), so the face crossings inside that cube, each of which would only
 * have moved the photon, become one step.  VOXEL steps at every voxel face, as
 * the reference does (src/mc3d_gpu.cu:181-339).  Both are the reference's
 * physics, including the weight its end-of-chunk quickfix removes
 * (src/mc3d_gpu.cu:343-353): a box holds one tissue and stops one voxel short of
 * any refractive-index change or top or lateral face, so every reflection
 * happens in a one-voxel step; only the step counts in mc3d_totals differ.  The
 * mode applies to fast and FP64 math; exact math always steps at every face, and
 * so does a launch with a geometry of nx * ny * (nz + 63) >= 2^32 voxels. */
enum mc3d_steps { MC3D_STEPS_MERGED = 0, MC3D_STEPS_VOXEL = 1 };

/* Voxel geometry (geometry_t, src/mc3d_types.h:38-43), tissue indices as uint8
 * after the reader's +1 remap (0 = air). */
typedef struct {
    int32_t nx, ny, nz;
    int32_t pad;
    double dx, dy, dz;      /* mm; stored as float on the device like geometry_t */
    const uint8_t *tissue;  /* nz*ny*nx, x fastest */
} mc3d_geom;

/* Optical properties (opticalprops_t, src/mc3d_types.h:28-36), index 0 = air. */
typedef struct {
    int32_t num_tissue_types; /* including air, 2 .. 256 */
    int32_t pad;
    const float *mua, *mus, *g, *n; /* 1/mm, 1/mm, -, - */
} mc3d_props;

/* One simulation.  Stream i (0 <= i < streams) draws from multiplier
 * table[1 + i mod (table_len - 1)] seeded as init_RNG does, and runs photons
 * i, i + streams, i + 2 streams, ... < photons. */
typedef struct {
    int32_t geom;     /* index into the geometry array */
    int32_t props;    /* index into the optical-property array */
    int32_t beam;     /* enum mc3d_beam */
    int32_t pad;
    int64_t photons;
    int64_t streams;  /* 0: min(photons, MC3D_DEFAULT_STREAMS), i.e. one photon per stream,
                         which balances a launch at photon granularity */
    uint64_t seed;    /* the reference's xinit; must satisfy init_RNG's check */
    int64_t stream_first; /* run only streams [stream_first, stream_first + stream_count): */
    int64_t stream_count; /* one shard of the job; 0 = all streams.  Shards' tallies add up
                             exactly to the whole job's */
} mc3d_job;

#define MC3D_DEFAULT_STREAMS (1ll << 40) /* the jump-ahead covers 2^40 seeding attempts */

/* Per-job totals.  Conservation, exact in integers:
 *   w_launched = r_in + r_out + t_in + t_out + absorbed + rr_killed - rr_created + lost */
typedef struct {
    uint64_t photons;    /* photons finished */
    uint64_t steps;      /* photon steps executed (iterations of src/mc3d_gpu.cu:175-340;
                            a merged step counts once) */
    uint64_t w_launched; /* sum Q(1 - Rsp) */
    uint64_t r_in;       /* reflected, inside the surface grid (= sum of drs bins) */
    uint64_t r_out;      /* reflected, outside the grid */
    uint64_t t_in;       /* frozen below the surface inside the grid (= sum of trans bins) */
    uint64_t t_out;
    uint64_t absorbed;
    uint64_t rr_killed;  /* weight removed by russian roulette */
    uint64_t rr_created; /* weight added to roulette survivors */
    uint64_t lost;       /* weight of photons killed by the NaN/db==0 quickfix or the step cap */
    uint64_t capped;     /* photons stopped by the per-photon step cap */
    uint64_t quickfix;   /* photons zeroed by the quickfix (src/mc3d_gpu.cu:343-353) */
    uint64_t fresnel;    /* Fresnel events (index-mismatched face crossings) */
} mc3d_totals;

/* Results of one job; bin arrays are nx*ny of the job's geometry (x fastest) and
 * may be NULL when not wanted. */
typedef struct {
    uint64_t *drs;     /* sum Q(W) of reflected photons per surface bin */
    uint64_t *drs_sq;  /* sum Q(W^2) per bin, for the per-bin variance */
    uint64_t *trans;   /* sum Q(W) of photons frozen below the surface */
    uint64_t *absorption; /* nz*ny*nx: sum Q(W_before) - Q(W_after) of every absorption in
                             the voxel (clamped into the grid, as the reference's disabled
                             tally, src/mc3d_gpu.cu:265-272); needs options.absorption_map */
    mc3d_totals totals;
} mc3d_out;

/* Per-photon final state, for debugging and parity tests. */
typedef struct {
    float x, y, z, ux, uy, uz, W, s;
    uint32_t steps;
    uint32_t tissue;
    uint64_t rng; /* packed generator state after the photon */
} mc3d_photon_record;

typedef struct {
    int32_t device;         /* CUDA device ordinal */
    int32_t math;           /* enum mc3d_math */
    int32_t block;          /* threads per block, 0 = tuned */
    int32_t blocks_per_sm;  /* 0 = as many as fit */
    int32_t absorption_map; /* 1: tally absorbed weight per voxel (sum over voxels = absorbed) */
    int32_t use_graph;      /* 1: a plan's first execute captures the tally clear and the
                               launch into a CUDA graph, later executes replay it */
    int64_t max_steps;      /* per-photon step cap, 0 = 2^24 */
    mc3d_photon_record *photon_log; /* host, sum of photons over jobs, or NULL */
    volatile int32_t *cancel;       /* optional host flag, read when a stream starts */
    int32_t steps;                  /* enum mc3d_steps (fast and FP64 math) */
    int32_t pad;
} mc3d_options;

/* ------------------------------------------------------------------ engine */

const char *mc3d_last_error(void);
int mc3d_abi_version(void);
void mc3d_default_options(mc3d_options *opt);

/* Run every job in one persistent launch and fill out[0..njobs-1].
 * Replaces run_3dmc_gpu (src/mc3d_gpu.cu:388-601). */
int mc3d_run(const mc3d_geom *geoms, int32_t ngeoms, const mc3d_props *props, int32_t nprops,
             const mc3d_job *jobs, int32_t njobs, const uint32_t *table, int64_t table_len,
             const mc3d_options *opt, mc3d_out *out);

/* Reusable plan: inputs uploaded once, then executed any number of times.
 * execute() is asynchronous on `stream` (a cudaStream_t, NULL = the plan's own).
 * Plans (and mc3d_run) take their device memory from a pool private to the
 * library, one per device; destroy() waits for the device and returns the memory
 * to that pool, which keeps up to 4 GiB of it for the next plan and hands the rest
 * back to the driver. */
typedef struct mc3d_plan mc3d_plan;
int mc3d_plan_create(mc3d_plan **plan, const mc3d_geom *geoms, int32_t ngeoms,
                     const mc3d_props *props, int32_t nprops, const mc3d_job *jobs,
                     int32_t njobs, const uint32_t *table, int64_t table_len,
                     const mc3d_options *opt);
int mc3d_plan_execute(mc3d_plan *plan, void *stream);
int mc3d_plan_read(mc3d_plan *plan, mc3d_out *out);
/* launch shape picked for the plan: threads per block, blocks, dynamic smem bytes */
int mc3d_plan_shape(const mc3d_plan *plan, int32_t *block, int32_t *grid, int32_t *smem);
/* device pointer of the first per-job totals (njobs * 14 uint64), for in-device checks */
int mc3d_plan_device_totals(const mc3d_plan *plan, void **ptr);
void mc3d_plan_destroy(mc3d_plan *plan);

/* The packed initial generator state and multiplier of streams [first, first+count)
 * of job `job`, computed on the GPU (for parity tests against init_RNG). */
int mc3d_stream_seeds(const mc3d_job *job, const uint32_t *table, int64_t table_len,
                      int64_t first, int64_t count, uint64_t *x_out, uint32_t *a_out,
                      int32_t device);

/* n draws of rand_MWC_co (gpumcml_rng/gpumcml_rng.cu:38-46) per generator, computed
 * on the GPU: out[g * n + d] for generator g of ngen with states x[g], a[g]. */
int mc3d_mwc_draws(const uint64_t *x, const uint32_t *a, int64_t ngen, int64_t n, float *out,
                   int32_t device);

/* No counterpart in the reference: the safe-distance map behind MC3D_STEPS_MERGED,
 * computed on the GPU from a host grid (for tests).  radius holds nz + 63 slices
 * of nx * ny (x fastest): slices below the grid stand for the medium's
 * continuation there (the voxel index is clamped).  radius[v] is the largest
 * r <= 63 such that every voxel within Chebyshev distance r of v has v's tissue
 * and lies below the top face and inside the lateral faces. */
int mc3d_safe_distance(const uint8_t *tissue, int32_t nx, int32_t ny, int32_t nz,
                       uint8_t *radius, int32_t device);

/* ------------------------------------------------- allocation-free entry point */

/* No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc -- code inside a framework whose caching allocator owns the device
 * memory (a raw cudaMalloc/cudaFree there synchronises the device and fragments
 * the framework's pool), or a loop with a fixed memory budget.
 *
 * Runs one job (fast math) like mc3d_run, allocating nothing.  geom->tissue and
 * the four outputs are DEVICE pointers the caller owns: drs, drs_sq and trans hold
 * nx*ny words, totals the 14 words of mc3d_totals in its order; all four are
 * overwritten.  props and table are host arrays.  The launch's working memory
 * (descriptors, optical table, multipliers, rejection list, work counter) is one
 * static device array of MC3D_NOALLOC_SCRATCH_BYTES that every GPU loading the
 * library holds until exit; inputs beyond its limits return MC3D_ERR_CAPACITY.
 * All calls share that array: calls whose work overlaps on the GPU race, so run
 * them one after another.  Before its launch the call synchronises `stream` (it
 * reads back the grid's largest tissue index and the seeding scan), so the host
 * waits for the work already queued there; it returns once the photon kernel is
 * queued.  The first call on a device looks up the array's address and should
 * come before any stream capture.  The caller's current device is restored. */
#define MC3D_NOALLOC_SCRATCH_BYTES (1u << 20)
#define MC3D_NOALLOC_MAX_TABLE 230401     /* safe-prime table lines */
#define MC3D_NOALLOC_MAX_TISSUES 256
#define MC3D_NOALLOC_MAX_REJECTIONS 4096  /* rejected seeding attempts in the job */
int mc3d_run_noalloc(const mc3d_geom *geom, const mc3d_props *props, const mc3d_job *job,
                     const uint32_t *table, int64_t table_len, int32_t device, void *stream,
                     uint64_t *drs, uint64_t *drs_sq, uint64_t *trans, uint64_t *totals);

/* ----------------------------------------------- reference-shaped entry point */

/* Layout-compatible with geometry_t and opticalprops_t (src/mc3d_types.h:28-43). */
typedef struct {
    float sample_dx, sample_dy, sample_dz;
    float length_x, length_y, length_z;
    int num_x, num_y, num_z;
    int *tissue_type; /* after the reader's remap, 0 = air */
} mc3d_ref_geometry;

typedef struct {
    int num_tissue_types;
    float *n, *mua, *mus, *g;
    int alloc_where;
} mc3d_ref_opticalprops;

/* Same arguments and meaning as run_3dmc_gpu (src/mc3d_gpu.cu:388): R and T are
 * accumulated with the un-normalised reflected / transmitted weight per bin,
 * *num_finished_photons is set.  R_tot / T_tot receive the totals inside and
 * outside the grid (the reference leaves them untouched); A is left untouched as
 * in the reference.  The seed is time(NULL) unless MC3D_SEED is set, the table is
 * ./safeprimes_base32.txt as in src/mc3d_rng.cu:16.  Returns a status instead of
 * exiting. */
int mc3d_run_3dmc_gpu(mc3d_ref_geometry geometry, mc3d_ref_opticalprops optProps,
                      int num_photons, double *R, double *R_tot, double *T, double *T_tot,
                      float *A, int *num_finished_photons);

/* ------------------------------------------------------------ safe primes */

/* n multipliers a < below (descending), each with a*2^32-1 and a*2^31-1 prime
 * (the multiply-with-carry condition behind safeprimes_base32.txt, whose file is
 * not distributed with the reference).  below = 0 means 2^32. */
int mc3d_safeprime_table(uint32_t *out, int64_t n, uint64_t below, int32_t threads);
/* write / read the reference's text format: one "a hi lo" line per multiplier,
 * where hi:lo is a*2^32-1; only the first column is read (gpumcml_rng.cu:80,97) */
int mc3d_safeprimes_write(const char *path, const uint32_t *table, int64_t n);
int mc3d_safeprimes_read(const char *path, uint32_t *out, int64_t cap, int64_t *n_read);

/* ------------------------------------------------------------------- files */

/* Geometry file (src/mc3d_io.cu:107-169): int32 3, int32 nx, ny, nz, double dx, dy, dz,
 * int32 tissue[nz][ny][nx].  Values are remapped +1 with 256 -> 0 (air). */
int mc3d_read_geometry_header(const char *path, int32_t *nx, int32_t *ny, int32_t *nz,
                              double *dx, double *dy, double *dz);
int mc3d_read_geometry(const char *path, uint8_t *tissue, int64_t cap);
/* Optical-property file (src/mc3d_io.cu:16-66): int32 T, then T records of double
 * mua, mus, g, n.  Air (0, 0, 0, 1) is prepended; *num_tissue_types = T + 1. */
int mc3d_read_optprops(const char *path, int32_t *num_tissue_types, float *mua, float *mus,
                       float *g, float *n, int32_t cap);
/* save_property (src/mc3d_io.cu:175-216): int32 dims, int32 nx, ny[, nz],
 * double dx, dy[, dz], double data[]. */
int mc3d_save_property(const char *path, int32_t dims, int32_t nx, int32_t ny, int32_t nz,
                       double dx, double dy, double dz, const double *data);
/* save_diff_refl (src/mc3d_io.cu:218-227): <outname>_drs.bin = R / num_photons */
int mc3d_save_diff_refl(const char *outname, int32_t nx, int32_t ny, double dx, double dy,
                        const double *R, int64_t num_photons);

#ifdef __cplusplus
}
#endif

#endif /* MC3D_H */
