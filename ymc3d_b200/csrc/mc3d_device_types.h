/*
 * mc3d_device_types.h -- launch descriptors shared by the host driver and the
 * photon kernel.  One launch covers any number of jobs; each job names a geometry
 * and an optical-property set and owns a contiguous range of global stream
 * indices and of tally bins.
 */
#ifndef MC3D_DEVICE_TYPES_H
#define MC3D_DEVICE_TYPES_H

#include <stdint.h>
#include <cuda_runtime.h>
#include "mc3d_rng.h"

/* order of the per-job totals (matches mc3d_totals in include/mc3d.h) */
#define MC3D_NUM_TOTALS 14

/* largest safe distance of the merged-step map, and the number of slices the
 * map adds below the grid (the clamped continuation of the medium) */
#define MC3D_SAFE_CAP 63

namespace mc3d {

struct GeomDev {
    int nx, ny, nz, pad;
    float dx, dy, dz;      /* voxel size, float as in geometry_t (src/mc3d_types.h:38-43) */
    float Lx, Ly, Lz;      /* voxel size * count, computed in float */
    float rdx, rdy, rdz;   /* 1 / voxel size (fast math only) */
    float pad2;
    const uint8_t *tissue; /* nz*ny*nx, x fastest; 0 = air */
    const uint16_t *cells; /* tissue | box radius << 8, nz + MC3D_SAFE_CAP slices (merged) */
};

struct JobDev {
    int64_t stream_base; /* first global stream index of the job's launched range */
    int64_t stream_first; /* job-local index of that first stream (shards) */
    int64_t streams;     /* S, the job's total stream count */
    int64_t stream_base_end; /* stream_base + streams launched */
    int64_t scan_base;   /* first index of the job in the seeding scan, which covers
                            streams [0, stream_first + launched) */
    int64_t per_stream;  /* floor(photons / S) */
    int64_t remainder;   /* photons mod S: streams below it run one extra photon */
    int64_t bin_offset;  /* first tally bin */
    int64_t photon_base; /* first record of the optional photon log */
    int64_t amap_offset; /* first voxel of the job in the absorption map */
    uint64_t seed;       /* seeding-generator start (the reference's xinit) */
    int32_t geom;
    int32_t props_offset; /* first float4 of the job's optical table in shared memory */
    int32_t beam;         /* 0 uniform over the top face, 1 pencil at the centre */
    int32_t rej_offset;   /* slice of the rejection list */
    int32_t rej_count;
    int32_t pad;
};

/* A stream whose seeding attempt(s) were rejected (gpumcml_rng/gpumcml_rng.cu:100)
 * and the running total of rejected attempts up to and including it; every later
 * stream of the job starts that many attempts further along. */
struct RejectionDev {
    int64_t stream;
    int64_t cum;
};

struct PhotonRecord {
    float x, y, z, ux, uy, uz, W, s;
    uint32_t steps;
    uint32_t tissue;
    uint64_t rng;
};

struct KernelParams {
    const JobDev *jobs;
    const GeomDev *geoms;
    const float4 *props_table; /* 3 float4 per tissue (see photon_step), sets back to back */
    const uint32_t *multipliers; /* safe-prime table, entry 0 = seeding multiplier */
    const RejectionDev *rejections;
    unsigned long long *drs;    /* sum Q(W) of reflected photons per surface bin */
    unsigned long long *drs_sq; /* sum Q(W^2) */
    unsigned long long *trans;  /* sum Q(W) of photons frozen below the surface */
    unsigned long long *totals; /* njobs * MC3D_NUM_TOTALS */
    unsigned long long *amap;   /* sum Q(dW) per voxel (absorption map variant only) */
    unsigned long long *work_counter;
    const int *cancel;
    PhotonRecord *photon_log;
    int64_t num_multipliers;
    uint64_t mult_magic;      /* floor((2^64 - 1) / (num_multipliers - 1)), see stream_multiplier */
    int64_t total_streams;
    int64_t max_steps;
    int32_t njobs;
    int32_t props_entries;
    int32_t ngeoms;
    int32_t pad_geoms;
    mc3d_seed_consts seed;
    GeomDev geom0; /* the only geometry of a one-geometry launch, read from the
                      parameter space instead of being copied per thread */
};

} /* namespace mc3d */

#endif /* MC3D_DEVICE_TYPES_H */
