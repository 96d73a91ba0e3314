/*
 * mc3d_kernel_f64.cu -- the photon kernel stepping in FP64 (MC3D_MATH_F64).
 * Built with -fmad=false -prec-div=true -prec-sqrt=true.  Every transport
 * quantity is a double; the loop, its quirks and the random numbers are those of
 * the FP32 kernels, one step per voxel face.  It is the precision reference the
 * FP32 results are stated against.
 */
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

namespace mc3d {

__global__ void __launch_bounds__(256, 2) photon_kernel_f64(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathF64, false>(P);
}

/* with the per-voxel absorption map */
__global__ void __launch_bounds__(256, 2)
    photon_kernel_f64_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathF64, true>(P);
}

cudaError_t launch_photon_f64(const KernelParams &P, int grid, int block, size_t smem,
                              cudaStream_t stream)
{
    if (P.amap) photon_kernel_f64_amap<<<grid, block, smem, stream>>>(P);
    else photon_kernel_f64<<<grid, block, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t occupancy_photon_f64(int block, size_t smem, int *blocks_per_sm)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, photon_kernel_f64, block,
                                                         smem);
}

cudaError_t smem_limit_photon_f64(size_t smem)
{
    cudaError_t e = cudaFuncSetAttribute(photon_kernel_f64,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(photon_kernel_f64_amap,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

cudaError_t attributes_photon_f64(cudaFuncAttributes *attr)
{
    return cudaFuncGetAttributes(attr, photon_kernel_f64);
}

} /* namespace mc3d */
