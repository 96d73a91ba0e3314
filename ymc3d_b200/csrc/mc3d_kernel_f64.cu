/*
 * mc3d_kernel_f64.cu -- the photon kernel stepping in FP64 (MC3D_MATH_F64).
 * Built with -fmad=false -prec-div=true -prec-sqrt=true.  Every transport
 * quantity is a double; the loop, its quirks and the random numbers are those of
 * the FP32 kernels, with one step per voxel face or merged steps (the step mode
 * of the plan).  It is the precision reference the FP32 results are stated
 * against.
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

/* merged steps over the packed cell map */
__global__ void __launch_bounds__(256, 2)
    photon_kernel_f64_merged(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathF64, false, true>(P);
}

__global__ void __launch_bounds__(256, 2)
    photon_kernel_f64_merged_amap(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathF64, true, true>(P);
}

typedef void (*photon_kernel_t)(KernelParams);

static photon_kernel_t pick(bool amap, int variant)
{
    if (variant & MC3D_VARIANT_VOXEL_STEPS) return amap ? photon_kernel_f64_amap : photon_kernel_f64;
    return amap ? photon_kernel_f64_merged_amap : photon_kernel_f64_merged;
}

cudaError_t launch_photon_f64(const KernelParams &P, int grid, int block, size_t smem,
                              cudaStream_t stream, int variant)
{
    pick(P.amap != nullptr, variant)<<<grid, block, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t occupancy_photon_f64(int block, size_t smem, int *blocks_per_sm, int variant)
{
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, pick(false, variant),
                                                         block, smem);
}

cudaError_t smem_limit_photon_f64(size_t smem)
{
    const photon_kernel_t all[] = {photon_kernel_f64, photon_kernel_f64_amap,
                                   photon_kernel_f64_merged, photon_kernel_f64_merged_amap};
    for (photon_kernel_t k : all) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t attributes_photon_f64(cudaFuncAttributes *attr)
{
    return cudaFuncGetAttributes(attr, photon_kernel_f64);
}

} /* namespace mc3d */
