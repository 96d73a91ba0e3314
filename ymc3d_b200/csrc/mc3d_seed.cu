/*
 * mc3d_seed.cu -- stream seeding on the GPU.
 *
 * init_RNG (gpumcml_rng/gpumcml_rng.cu:59-118) seeds its streams one after
 * another from a single seeding generator.  Here every stream jumps straight to
 * its own seeding attempt (mc3d_seed_jump), so seeding is parallel and needs no
 * per-stream state in memory.  The only sequential coupling is a rejected attempt,
 * which shifts every later stream by one attempt; the scan below finds the first
 * rejected stream of each job and the host lists the (rare) rejections from there.
 */
#include <climits>
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

namespace mc3d {

__global__ void seed_scan_kernel(const JobDev *jobs, int njobs, const uint32_t *mult,
                                 int64_t nmult, const __grid_constant__ mc3d_seed_consts sc,
                                 int64_t total_streams, unsigned long long *first_reject)
{
    for (int64_t gs = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; gs < total_streams;
         gs += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = njobs - 1; /* job whose scan range holds gs */
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (jobs[mid].scan_base <= gs) lo = mid;
            else hi = mid - 1;
        }
        int j = lo;
        int64_t local = gs - jobs[j].scan_base;
        uint32_t fora = mult[1 + (local % (nmult - 1))];
        uint64_t xs = mc3d_seed_jump(&sc, jobs[j].seed, (uint64_t)local);
        uint64_t st = mc3d_seed_attempt(xs, sc.begin, fora);
        if (!mc3d_seed_valid(st, fora)) atomicMin(first_reject + j, (unsigned long long)local);
    }
}

cudaError_t launch_seed_scan(const JobDev *jobs, int njobs, const uint32_t *mult, int64_t nmult,
                             const mc3d_seed_consts &sc, int64_t total_streams,
                             unsigned long long *first_reject, cudaStream_t stream)
{
    if (total_streams <= 0) return cudaSuccess;
    int block = 256;
    int64_t want = (total_streams + block - 1) / block;
    int grid = (int)(want < 148 * 64 ? want : 148 * 64);
    seed_scan_kernel<<<grid, block, 0, stream>>>(jobs, njobs, mult, nmult, sc, total_streams,
                                                 first_reject);
    return cudaGetLastError();
}

__global__ void seed_dump_kernel(const __grid_constant__ KernelParams P, int64_t first,
                                 int64_t count, uint64_t *x_out, uint32_t *a_out)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const JobDev &jb = P.jobs[0];
    int64_t local = first + t;
    uint32_t fora = P.multipliers[1 + (local % (P.num_multipliers - 1))];
    x_out[t] = stream_seed(P, jb, local, fora);
    a_out[t] = fora;
}

cudaError_t launch_seed_dump(const KernelParams &P, int64_t first, int64_t count,
                             uint64_t *x_out, uint32_t *a_out, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    int block = 256;
    int grid = (int)((count + block - 1) / block);
    seed_dump_kernel<<<grid, block, 0, stream>>>(P, first, count, x_out, a_out);
    return cudaGetLastError();
}

__global__ void mwc_draws_kernel(const uint64_t *x, const uint32_t *a, int64_t ngen, int64_t n,
                                 float *out)
{
    int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngen) return;
    uint64_t st = x[g];
    uint32_t m = a[g];
    for (int64_t d = 0; d < n; d++) out[g * n + d] = mc3d_rand_co(&st, m);
}

cudaError_t launch_mwc_draws(const uint64_t *x, const uint32_t *a, int64_t ngen, int64_t n,
                             float *out, cudaStream_t stream)
{
    if (ngen <= 0 || n <= 0) return cudaSuccess;
    int block = 256;
    int grid = (int)((ngen + block - 1) / block);
    mwc_draws_kernel<<<grid, block, 0, stream>>>(x, a, ngen, n, out);
    return cudaGetLastError();
}

} /* namespace mc3d */
