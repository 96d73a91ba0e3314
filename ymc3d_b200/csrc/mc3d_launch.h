/*
 * mc3d_launch.h -- launchers of the device code, one per translation unit.
 * The fast and exact photon kernels live in separate files because their math
 * depends on compile flags (-use_fast_math vs -fmad=false).
 */
#ifndef MC3D_LAUNCH_H
#define MC3D_LAUNCH_H

#include <cuda_runtime.h>
#include "mc3d_device_types.h"

namespace mc3d {

/* fast kernel variant bits: one step per voxel face instead of merged steps.
 * (A 64-register build of 4 blocks of 256 per SM measured 2-12 % slower than the
 * 80-register one and is not built: one kernel serves every launch shape, so the
 * tallies cannot depend on the shape.) */
#define MC3D_VARIANT_VOXEL_STEPS 2
/* one geometry in the launch: its descriptor is read from the kernel parameters */
#define MC3D_VARIANT_ONE_GEOM 4
cudaError_t launch_photon_fast(const KernelParams &P, int grid, int block, size_t smem,
                               cudaStream_t stream, int variant);
cudaError_t launch_photon_exact(const KernelParams &P, int grid, int block, size_t smem,
                                cudaStream_t stream);
cudaError_t launch_photon_f64(const KernelParams &P, int grid, int block, size_t smem,
                              cudaStream_t stream, int variant);
cudaError_t occupancy_photon_fast(int block, size_t smem, int *blocks_per_sm, int variant);
cudaError_t occupancy_photon_f64(int block, size_t smem, int *blocks_per_sm, int variant);
cudaError_t smem_limit_photon_f64(size_t smem);
cudaError_t attributes_photon_f64(cudaFuncAttributes *attr);
cudaError_t occupancy_photon_exact(int block, size_t smem, int *blocks_per_sm);
cudaError_t smem_limit_photon_fast(size_t smem);
cudaError_t smem_limit_photon_exact(size_t smem);
cudaError_t attributes_photon_fast(cudaFuncAttributes *attr);
cudaError_t attributes_photon_exact(cudaFuncAttributes *attr);

/* first rejected seeding attempt per job, assuming none before it (UINT64_MAX if none) */
cudaError_t launch_seed_scan(const JobDev *jobs, int njobs, const uint32_t *mult,
                             int64_t nmult, const mc3d_seed_consts &sc, int64_t total_streams,
                             unsigned long long *first_reject, cudaStream_t stream);
/* states of streams [first, first+count) of job 0 of `jobs` */
cudaError_t launch_seed_dump(const KernelParams &P, int64_t first, int64_t count,
                             uint64_t *x_out, uint32_t *a_out, cudaStream_t stream);
/* safe-distance map of a tissue grid (merged steps): out, tmp_a and tmp_b hold
 * nx * ny * (nz + MC3D_SAFE_CAP) bytes each */
cudaError_t launch_safe_distance(const uint8_t *tissue, int nx, int ny, int nz, uint8_t *out,
                                 uint8_t *tmp_a, uint8_t *tmp_b, cudaStream_t stream);
/* packed cells (tissue | box radius << 8) from the safe distances of the tissue grid
 * (radius) and of its refractive-index classes (radius_n; the same map when every
 * tissue has its own class) */
cudaError_t launch_pack_cells(const uint8_t *tissue, const uint8_t *radius,
                              const uint8_t *radius_n, int nx, int ny, int nz, uint16_t *cells,
                              cudaStream_t stream);
/* out[v] = classes[tissue[v]] for nv voxels (classes: 256 entries, host memory) */
cudaError_t launch_index_classes(const uint8_t *tissue, int64_t nv, const uint8_t *classes,
                                 uint8_t *out, cudaStream_t stream);
cudaError_t launch_mwc_draws(const uint64_t *x, const uint32_t *a, int64_t ngen, int64_t n,
                             float *out, cudaStream_t stream);

} /* namespace mc3d */

#endif
