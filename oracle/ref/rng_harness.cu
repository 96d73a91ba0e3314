/*
 * rng_harness.cu -- C entry points into the reference's own RNG code.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled against gpumcml_rng/gpumcml_rng.cu where
 * it lies (included below, not copied): init_RNG runs on the host, rand_MWC_co
 * runs in a test kernel on the GPU.
 */
#include <cstring>
#include <cstdint>
#include "gpumcml_rng.cu"

extern "C" int ref_init_rng(UINT64 *x, UINT32 *a, UINT32 n, const char *file, UINT64 xinit)
{
    return init_RNG(x, a, n, file, xinit);
}

__global__ void ref_draws_kernel(UINT64 *x, UINT32 *a, int ngen, int n, float *out)
{
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngen) return;
    UINT64 st = x[g];
    UINT32 m = a[g];
    for (int d = 0; d < n; d++) out[(size_t)g * n + d] = rand_MWC_co(&st, &m);
}

/* n draws of rand_MWC_co for each of ngen generators; 0 on success */
extern "C" int ref_mwc_draws(const UINT64 *x, const UINT32 *a, int ngen, int n, float *out)
{
    UINT64 *dx = 0;
    UINT32 *da = 0;
    float *dout = 0;
    int rc = 1;
    if (cudaMalloc(&dx, sizeof(UINT64) * ngen) != cudaSuccess) goto done;
    if (cudaMalloc(&da, sizeof(UINT32) * ngen) != cudaSuccess) goto done;
    if (cudaMalloc(&dout, sizeof(float) * (size_t)ngen * n) != cudaSuccess) goto done;
    cudaMemcpy(dx, x, sizeof(UINT64) * ngen, cudaMemcpyHostToDevice);
    cudaMemcpy(da, a, sizeof(UINT32) * ngen, cudaMemcpyHostToDevice);
    ref_draws_kernel<<<(ngen + 255) / 256, 256>>>(dx, da, ngen, n, dout);
    if (cudaMemcpy(out, dout, sizeof(float) * (size_t)ngen * n, cudaMemcpyDeviceToHost) ==
        cudaSuccess)
        rc = 0;
done:
    cudaFree(dx);
    cudaFree(da);
    cudaFree(dout);
    return rc;
}

/* rand_MWC_co with a = 1 returns the conversion of the state's low word: compare
 * it with u32 -> float (toward zero) * 2^-32 for every u in [lo, hi); returns the
 * number of mismatches */
__global__ void ref_conv_kernel(unsigned long long lo, unsigned long long hi,
                                unsigned long long *bad)
{
    for (unsigned long long u = lo + blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
         u < hi; u += (unsigned long long)gridDim.x * blockDim.x) {
        UINT64 st = u;
        UINT32 one = 1;
        float r = rand_MWC_co(&st, &one);
        float e = __uint2float_rz((unsigned)u) * 0x1p-32f;
        if (__float_as_uint(r) != __float_as_uint(e)) atomicAdd(bad, 1ull);
    }
}

extern "C" long long ref_conversion_mismatches(unsigned long long lo, unsigned long long hi)
{
    unsigned long long *d = 0, h = 0;
    if (cudaMalloc(&d, sizeof h) != cudaSuccess) return -1;
    cudaMemset(d, 0, sizeof h);
    ref_conv_kernel<<<148 * 8, 256>>>(lo, hi, d);
    if (cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) h = (unsigned long long)-1;
    cudaFree(d);
    return (long long)h;
}
