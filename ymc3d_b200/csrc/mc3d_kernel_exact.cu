/*
 * mc3d_kernel_exact.cu -- the photon kernel with reproducible IEEE math.
 * Built with -fmad=false -prec-div=true -prec-sqrt=true: every operation is
 * correctly rounded and nothing is contracted, so a trajectory matches the CPU
 * transcription bit for bit.
 */
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

namespace mc3d {

__global__ void __launch_bounds__(256, 3) photon_kernel_exact(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathExact, false>(P);
}

/* with the per-voxel absorption map */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_exact_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathExact, true>(P);
}

cudaError_t launch_photon_exact(const KernelParams &P, int grid, int block, size_t smem,
                                cudaStream_t stream)
{
    if (P.amap) photon_kernel_exact_amap<<<grid, block, smem, stream>>>(P);
    else photon_kernel_exact<<<grid, block, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t occupancy_photon_exact(int block, size_t smem, int *blocks_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, photon_kernel_exact, block,
                                                         smem);
}

cudaError_t smem_limit_photon_exact(size_t smem)
{
    cudaError_t e = cudaFuncSetAttribute(photon_kernel_exact,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(photon_kernel_exact_amap,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t attributes_photon_exact(cudaFuncAttributes *attr)
{
    return cudaFuncGetAttributes(attr, photon_kernel_exact);
}

} /* namespace mc3d */
