/*
 * mc3d_kernel_fast.cu -- the photon kernel with the GPU's approximate math.
 * Built with -use_fast_math like the reference (CMakeLists.txt:18): divisions,
 * sqrtf, logf and sinf map to the approximate hardware paths.
 */
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

namespace mc3d {

__global__ void __launch_bounds__(256, 3) photon_kernel_fast(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false>(P);
}

/* with the per-voxel absorption map */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, true>(P);
}

/* 64-register budget: four blocks of 256 per SM, at the price of a few spills */
__global__ void __launch_bounds__(256, 4)
    photon_kernel_fast_r64(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false>(P);
}

/* the split step (photon_step_fast), kept for A/B measurements */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_fast_split(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, true>(P);
}

cudaError_t launch_photon_fast(const KernelParams &P, int grid, int block, size_t smem,
                                cudaStream_t stream, int variant)
{
    if (P.amap) photon_kernel_fast_amap<<<grid, block, smem, stream>>>(P);
    else if (variant == 1) photon_kernel_fast_r64<<<grid, block, smem, stream>>>(P);
    else if (variant == 2) photon_kernel_fast_split<<<grid, block, smem, stream>>>(P);
    else photon_kernel_fast<<<grid, block, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t occupancy_photon_fast(int block, size_t smem, int *blocks_per_sm, int variant)
{
    if (variant == 1)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm,
                                                             photon_kernel_fast_r64, block, smem);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, photon_kernel_fast, block,
                                                         smem);
}

cudaError_t smem_limit_photon_fast(size_t smem)
{
    cudaError_t e = cudaFuncSetAttribute(photon_kernel_fast,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(photon_kernel_fast_r64, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(photon_kernel_fast_split,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(photon_kernel_fast_amap,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t attributes_photon_fast(cudaFuncAttributes *attr)
{
    return cudaFuncGetAttributes(attr, photon_kernel_fast);
}

} /* namespace mc3d */
