/*
 * texture_shim.h -- lets the reference's mc3d_gpu.cu compile on CUDA 12.
 *
 * TEST INFRASTRUCTURE ONLY (oracle build of the reference binary).  CUDA 12
 * removed texture references; the reference declares one
 * (src/mc3d_gpu.cu:23), fetches it with tex3D (:25), fills its fields (:403,
 * :414-418) and binds it with cudaBindTextureToArray (:421).  This header,
 * force-included before that file, supplies a `texture` type with those fields,
 * a bind that creates an equivalent texture object (same channel, point filter,
 * clamp addressing, unnormalised coordinates) and a tex3D that reads it.  The
 * reference source itself is compiled unmodified, where it lies.
 */
#ifndef MC3D_REF_TEXTURE_SHIM_H
#define MC3D_REF_TEXTURE_SHIM_H

#include <cstring>
#include <cuda_runtime.h>
#include <texture_fetch_functions.h>

template <class T, int dim, enum cudaTextureReadMode mode>
struct texture {
    cudaChannelFormatDesc channelDesc;
    int normalized;
    enum cudaTextureFilterMode filterMode;
    enum cudaTextureAddressMode addressMode[3];
    texture() : channelDesc(cudaCreateChannelDesc<T>()), normalized(0),
                filterMode(cudaFilterModePoint)
    {
        addressMode[0] = addressMode[1] = addressMode[2] = cudaAddressModeClamp;
    }
};

static __device__ cudaTextureObject_t mc3d_ref_shim_tex;

template <class T, int dim, enum cudaTextureReadMode mode>
static cudaError_t cudaBindTextureToArray(const texture<T, dim, mode> &tex, cudaArray_const_t arr,
                                          const cudaChannelFormatDesc &)
{
    cudaResourceDesc res;
    memset(&res, 0, sizeof res);
    res.resType = cudaResourceTypeArray;
    res.res.array.array = (cudaArray_t)arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof td);
    for (int i = 0; i < 3; i++) td.addressMode[i] = tex.addressMode[i];
    td.filterMode = tex.filterMode;
    td.readMode = mode;
    td.normalizedCoords = tex.normalized;
    cudaTextureObject_t obj = 0;
    cudaError_t e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(mc3d_ref_shim_tex, &obj, sizeof obj);
}

#define tex3D(tex_, i_, j_, k_) tex3D<int>(mc3d_ref_shim_tex, (float)(i_), (float)(j_), (float)(k_))

#endif
