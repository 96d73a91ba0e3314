/*
 * mc3d_kernel_fast.cu -- the photon kernel with the GPU's approximate math.
 * Built with -use_fast_math like the reference (CMakeLists.txt:18): divisions,
 * sqrtf, logf and sinf map to the approximate hardware paths.
 */
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

namespace mc3d {

/* Eight instantiations: merged steps (box DDA over uniform cubes) or one step
 * per voxel face; with or without the absorption map; several geometries (their
 * descriptors in shared memory) or one (its descriptor read from the kernel
 * parameters, which keeps it out of the registers). */

/* merged steps */
__global__ void __launch_bounds__(256, 3) photon_kernel_fast(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, true>(P);
}

/* merged steps with the per-voxel absorption map */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, true, true>(P);
}

/* one step per voxel face, as the reference steps */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_voxel(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, false>(P);
}

__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_voxel_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, true, false>(P);
}

/* one geometry */
__global__ void __launch_bounds__(256, 3) photon_kernel_fast_g1(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, true, true>(P);
}

__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_amap_g1(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, true, true, true>(P);
}

__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_voxel_g1(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, false, true>(P);
}

__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_voxel_amap_g1(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, true, false, true>(P);
}

typedef void (*photon_kernel_t)(KernelParams);

static photon_kernel_t pick(bool amap, int variant)
{
    const bool voxel = (variant & MC3D_VARIANT_VOXEL_STEPS) != 0;
    if (variant & MC3D_VARIANT_ONE_GEOM) {
        if (amap) return voxel ? photon_kernel_fast_voxel_amap_g1 : photon_kernel_fast_amap_g1;
        return voxel ? photon_kernel_fast_voxel_g1 : photon_kernel_fast_g1;
    }
    if (amap) return voxel ? photon_kernel_fast_voxel_amap : photon_kernel_fast_amap;
    return voxel ? photon_kernel_fast_voxel : photon_kernel_fast;
}

cudaError_t launch_photon_fast(const KernelParams &P, int grid, int block, size_t smem,
                               cudaStream_t stream, int variant)
{
    pick(P.amap != nullptr, variant)<<<grid, block, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t occupancy_photon_fast(int block, size_t smem, int *blocks_per_sm, int variant)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pick(false, variant),
                                                         block, smem);
}

cudaError_t smem_limit_photon_fast(size_t smem)
{
    const photon_kernel_t all[] = {photon_kernel_fast,          photon_kernel_fast_amap,
                                   photon_kernel_fast_voxel,    photon_kernel_fast_voxel_amap,
                                   photon_kernel_fast_g1,       photon_kernel_fast_amap_g1,
                                   photon_kernel_fast_voxel_g1, photon_kernel_fast_voxel_amap_g1};
    for (photon_kernel_t k : all) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t attributes_photon_fast(cudaFuncAttributes *attr)
{
    return cudaFuncGetAttributes(attr, photon_kernel_fast);
}

} /* namespace mc3d */
