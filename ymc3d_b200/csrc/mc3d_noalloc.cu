/*
 * mc3d_noalloc.cu -- one job, no device allocation.
 *
 * mc3d_run and the plans allocate their working memory with cudaMalloc.  Some
 * callers cannot do that: code running inside a framework whose caching allocator
 * owns the device memory (a raw cudaMalloc/cudaFree pair there synchronises the
 * device and fragments the framework's pool), or a loop with a fixed memory
 * budget that must not grow at run time.  mc3d_run_noalloc serves them: the caller
 * passes the voxel grid and the output tallies in device memory it already owns,
 * and everything else the launch needs -- the job and geometry descriptors, the
 * optical table, the safe-prime multipliers, the seeding rejection list, the
 * stream work counter -- lives in one file-scope static device array of
 * MC3D_NOALLOC_SCRATCH_BYTES.  Every GPU that loads the library holds that array
 * until the process exits.
 *
 * The array is shared by all calls and keeps the last call's contents: each call
 * rewrites the descriptors and clears the counter before it launches, and two
 * calls whose work overlaps on the GPU race on it.  Host code never uses the
 * array's name as an address: on the first call on a device the entry point asks
 * cudaGetSymbolAddress for the device address (with that device current) and
 * keeps it; that first call should come before any stream capture.
 */
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mc3d.h"
#include "mc3d_engine.cuh"
#include "mc3d_launch.h"

/* host-side helpers of mc3d_api.cu (same library) */
namespace mc3d {
void set_last_error(const char *msg);
void make_seed_consts_host(uint32_t begin, mc3d_seed_consts *c);
int list_rejections_host(const mc3d_seed_consts &sc, uint64_t seed, const uint32_t *table,
                         int64_t table_len, int64_t streams, int64_t first,
                         std::vector<RejectionDev> &out, std::string *err);
}

namespace mc3d {
namespace {

/* layout of the static array (byte offsets, each 256-aligned) */
constexpr size_t kOffJob = 0;
constexpr size_t kOffGeom = 256;
constexpr size_t kOffProps = 512;
constexpr size_t kPropsBytes = 16ull * MC3D_TAB_STRIDE * MC3D_NOALLOC_MAX_TISSUES;
constexpr size_t kOffWords = kOffProps + ((kPropsBytes + 255) / 256) * 256;
constexpr size_t kWordsBytes = 256; /* counter, first rejection, max tissue */
constexpr size_t kOffRej = kOffWords + kWordsBytes;
constexpr size_t kRejBytes = sizeof(RejectionDev) * MC3D_NOALLOC_MAX_REJECTIONS;
constexpr size_t kOffMult = kOffRej + ((kRejBytes + 255) / 256) * 256;
constexpr size_t kMultBytes = 4ull * MC3D_NOALLOC_MAX_TABLE;
constexpr size_t kUsed = kOffMult + kMultBytes;
static_assert(kUsed <= MC3D_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout too large");
static_assert(sizeof(JobDev) <= 256 && sizeof(GeomDev) <= 256, "descriptor slots too small");

} /* namespace */

/* the scratch: one per GPU that loads the library, alive until exit */
static __device__ __align__(256) unsigned char g_noalloc_scratch[MC3D_NOALLOC_SCRATCH_BYTES];

/* one geometry, per-face steps; the descriptor is read from P.geom0 */
__global__ void __launch_bounds__(256, 3)
    photon_kernel_noalloc(const __grid_constant__ KernelParams P)
{
    photon_kernel_body<MathFast, false, false, true>(P);
}

/* largest tissue index of the device-resident grid, into a scratch word */
__global__ void noalloc_max_tissue_kernel(const uint8_t *grid, int64_t n, unsigned int *out)
{
    unsigned int m = 0;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
         v += (int64_t)gridDim.x * blockDim.x)
        m = max(m, (unsigned int)grid[v]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

} /* namespace mc3d */

using namespace mc3d;

namespace {

std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[64] = {nullptr};

int nfail(int code, const char *msg)
{
    mc3d::set_last_error(msg); /* read back with mc3d_last_error() */
    return code;
}

/* device address of the scratch on `device` (made current by the caller) */
int scratch_address(int device, unsigned char **out)
{
    if (device < 0 || device >= 64) return nfail(MC3D_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return nfail(MC3D_ERR_CUDA, cudaGetErrorString(e));
        g_scratch_ptr[device] = (unsigned char *)ptr;
    }
    *out = g_scratch_ptr[device];
    return MC3D_OK;
}

} /* namespace */


#define NA_TRY(call)                                                                          \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return nfail(MC3D_ERR_CUDA, cudaGetErrorString(e_));           \
    } while (0)

extern "C" int mc3d_run_noalloc(const mc3d_geom *geom, const mc3d_props *props,
                                const mc3d_job *job, const uint32_t *table, int64_t table_len,
                                int32_t device, void *stream, uint64_t *drs, uint64_t *drs_sq,
                                uint64_t *trans, uint64_t *totals)
{
    if (!geom || !props || !job || !table || !drs || !drs_sq || !trans || !totals ||
        !geom->tissue || !props->mua || !props->mus || !props->g || !props->n)
        return nfail(MC3D_ERR_ARG, "null argument");
    if (table_len < 2 || table_len > MC3D_NOALLOC_MAX_TABLE)
        return nfail(MC3D_ERR_CAPACITY, "table_len outside 2..MC3D_NOALLOC_MAX_TABLE");
    if (props->num_tissue_types < 2 || props->num_tissue_types > MC3D_NOALLOC_MAX_TISSUES)
        return nfail(MC3D_ERR_CAPACITY, "num_tissue_types outside 2..MC3D_NOALLOC_MAX_TISSUES");
    if (geom->nx <= 0 || geom->ny <= 0 || geom->nz <= 0 || !(geom->dx > 0) || !(geom->dy > 0) ||
        !(geom->dz > 0) || !std::isfinite(geom->dx) || !std::isfinite(geom->dy) ||
        !std::isfinite(geom->dz))
        return nfail(MC3D_ERR_GEOMETRY, "bad geometry size or voxel size");
    /* the same value checks as mc3d_plan_create: a non-finite coefficient would
     * step NaN positions and fill the tallies with garbage */
    for (int t = 0; t < props->num_tissue_types; t++)
        if (!std::isfinite(props->mua[t]) || !std::isfinite(props->mus[t]) ||
            !std::isfinite(props->g[t]) || !std::isfinite(props->n[t]))
            return nfail(MC3D_ERR_PROPS, "a tissue's optical property is not finite");
    for (int64_t i = 0; i < table_len; i++)
        if (table[i] < 2u) return nfail(MC3D_ERR_TABLE, "table holds a multiplier below 2");
    if (job->photons < 0 || job->streams < 0 || (job->beam != 0 && job->beam != 1))
        return nfail(MC3D_ERR_ARG, "bad photons/streams/beam");
    if (!mc3d_user_seed_valid(job->seed, table[0])) return nfail(MC3D_ERR_SEED, "not a valid seed");
    int64_t S = job->streams ? job->streams
                             : (job->photons < 1 ? 1
                                : (job->photons < MC3D_DEFAULT_STREAMS ? job->photons
                                                                       : MC3D_DEFAULT_STREAMS));
    int64_t first = job->stream_first;
    int64_t count = job->stream_count ? job->stream_count : S - first;
    if (first < 0 || count < 0 || first + count > S)
        return nfail(MC3D_ERR_ARG, "stream range outside the job");

    /* the caller's current device is put back on every return */
    int prev_device = 0;
    NA_TRY(cudaGetDevice(&prev_device));
    struct DeviceGuard {
        int prev;
        ~DeviceGuard() { cudaSetDevice(prev); }
    } guard{prev_device};
    NA_TRY(cudaSetDevice(device));
    unsigned char *base = nullptr;
    int st = scratch_address(device, &base);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;

    /* descriptors */
    const int nt = props->num_tissue_types;
    float4 tab[MC3D_TAB_STRIDE * MC3D_NOALLOC_MAX_TISSUES];
    for (int t = 0; t < nt; t++) {
        float mua = props->mua[t], mus = props->mus[t], g = props->g[t];
        volatile float mut = mua + mus;
        volatile float frac = mua / mut, rmut = 1.0f / mut, g2 = g * g, twog = 2 * g;
        volatile float inv2g = 1.0f / twog;
        tab[3 * t + 0] = make_float4(mua, mus, g, props->n[t]);
        tab[3 * t + 1] = make_float4(mut, frac, rmut, inv2g);
        tab[3 * t + 2] = make_float4(1 - g2, 1 - g, twog, 1 + g2);
    }
    GeomDev gd;
    memset(&gd, 0, sizeof gd);
    gd.nx = geom->nx; gd.ny = geom->ny; gd.nz = geom->nz;
    gd.dx = (float)geom->dx; gd.dy = (float)geom->dy; gd.dz = (float)geom->dz;
    gd.Lx = gd.dx * gd.nx; gd.Ly = gd.dy * gd.ny; gd.Lz = gd.dz * gd.nz;
    gd.rdx = 1.0f / gd.dx; gd.rdy = 1.0f / gd.dy; gd.rdz = 1.0f / gd.dz;
    gd.tissue = geom->tissue;
    JobDev jd;
    memset(&jd, 0, sizeof jd);
    jd.stream_base = 0;
    jd.stream_first = first;
    jd.streams = S;
    jd.stream_base_end = count;
    jd.scan_base = 0;
    jd.per_stream = job->photons / S;
    jd.remainder = job->photons % S;
    jd.seed = job->seed;
    jd.beam = job->beam;

    unsigned long long *words = (unsigned long long *)(base + kOffWords);
    const int64_t nb = (int64_t)geom->nx * geom->ny;
    NA_TRY(cudaMemcpyAsync(base + kOffProps, tab, sizeof(float4) * MC3D_TAB_STRIDE * nt,
                           cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + kOffGeom, &gd, sizeof gd, cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + kOffJob, &jd, sizeof jd, cudaMemcpyHostToDevice, s));
    NA_TRY(cudaMemcpyAsync(base + kOffMult, table, 4 * (size_t)table_len, cudaMemcpyHostToDevice,
                           s));
    /* the counter and the max-tissue word start at zero, the first rejection at "none" */
    NA_TRY(cudaMemsetAsync(words, 0, kWordsBytes, s));
    NA_TRY(cudaMemsetAsync(words + 1, 0xff, sizeof(unsigned long long), s));
    NA_TRY(cudaMemsetAsync(drs, 0, sizeof(uint64_t) * nb, s));
    NA_TRY(cudaMemsetAsync(drs_sq, 0, sizeof(uint64_t) * nb, s));
    NA_TRY(cudaMemsetAsync(trans, 0, sizeof(uint64_t) * nb, s));
    NA_TRY(cudaMemsetAsync(totals, 0, sizeof(uint64_t) * MC3D_NUM_TOTALS, s));

    /* every voxel's tissue must exist in the optical table */
    const int64_t nv = nb * geom->nz;
    noalloc_max_tissue_kernel<<<148 * 4, 256, 0, s>>>(geom->tissue, nv,
                                                       (unsigned int *)(words + 2));
    NA_TRY(cudaGetLastError());
    mc3d_seed_consts sc;
    make_seed_consts_host(table[0], &sc);
    NA_TRY(launch_seed_scan((const JobDev *)(base + kOffJob), 1, (const uint32_t *)(base + kOffMult),
                            table_len, sc, first + count, words + 1, s));
    unsigned long long hw[3];
    NA_TRY(cudaMemcpyAsync(hw, words, sizeof hw, cudaMemcpyDeviceToHost, s));
    NA_TRY(cudaStreamSynchronize(s));
    if ((int64_t)(unsigned int)hw[2] >= nt)
        return nfail(MC3D_ERR_TISSUE_RANGE, "the grid uses a tissue type the optical set lacks");
    if (hw[1] != ULLONG_MAX) {
        std::vector<RejectionDev> rej;
        std::string err;
        st = list_rejections_host(sc, job->seed, table, table_len, first + count,
                                  (int64_t)hw[1], rej, &err);
        if (st) return nfail(st, err.c_str());
        if ((int64_t)rej.size() > MC3D_NOALLOC_MAX_REJECTIONS)
            return nfail(MC3D_ERR_CAPACITY, "more rejected seeding attempts than "
                                            "MC3D_NOALLOC_MAX_REJECTIONS");
        jd.rej_count = (int32_t)rej.size();
        NA_TRY(cudaMemcpyAsync(base + kOffRej, rej.data(), sizeof(RejectionDev) * rej.size(),
                               cudaMemcpyHostToDevice, s));
        NA_TRY(cudaMemcpyAsync(base + kOffJob, &jd, sizeof jd, cudaMemcpyHostToDevice, s));
        NA_TRY(cudaStreamSynchronize(s)); /* jd and rej are host stack memory */
    }

    KernelParams P;
    memset(&P, 0, sizeof P);
    P.jobs = (const JobDev *)(base + kOffJob);
    P.geoms = (const GeomDev *)(base + kOffGeom);
    P.geom0 = gd;
    P.props_table = (const float4 *)(base + kOffProps);
    P.multipliers = (const uint32_t *)(base + kOffMult);
    P.rejections = (const RejectionDev *)(base + kOffRej);
    P.drs = (unsigned long long *)drs;
    P.drs_sq = (unsigned long long *)drs_sq;
    P.trans = (unsigned long long *)trans;
    P.totals = (unsigned long long *)totals;
    P.work_counter = words;
    P.num_multipliers = table_len;
    P.mult_magic = UINT64_MAX / (uint64_t)(table_len - 1);
    P.total_streams = count;
    P.max_steps = 1 << 24;
    P.njobs = 1;
    P.props_entries = MC3D_TAB_STRIDE * nt;
    P.seed = sc;
    int sms = 0, bps = 0;
    NA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    size_t smem = sizeof(float4) * P.props_entries;
    NA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, photon_kernel_noalloc, 256, smem));
    if (bps <= 0) return nfail(MC3D_ERR_CAPACITY, "kernel does not fit an SM");
    photon_kernel_noalloc<<<sms * bps, 256, smem, s>>>(P);
    NA_TRY(cudaGetLastError());
    return MC3D_OK;
}
