/*
 * mc3d_api.cu -- host driver behind the C ABI (include/mc3d.h).
 *
 * Replaces run_3dmc_gpu (src/mc3d_gpu.cu:388-601).  Where the reference loops on
 * the host -- back up the photon arrays, relaunch 45-step kernels, copy 230,400
 * slots back and tally reflectance with OpenMP every iteration -- a plan here
 * uploads the inputs once and runs a single persistent kernel that refills its own
 * photon slots and tallies on the device; the host reads the tallies back once.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mc3d.h"
#include "mc3d_launch.h"

using namespace mc3d;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return fail(MC3D_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));             \
    } while (0)

/* Plans take their device memory from a pool private to the library, one per
 * device, by stream-ordered allocation on the plan's stream.  The pool keeps up to
 * kPoolKeep bytes of freed memory, so a caller that runs plan after plan (one
 * mc3d_run per wavelength, say) reuses it instead of handing it back to the driver
 * and having it mapped again; a cudaFree of one plan's buffers took anywhere from
 * 2 to 260 ms.  Freed memory beyond kPoolKeep goes back at the next
 * synchronisation. */
const uint64_t kPoolKeep = 4ull << 30;
const int kMaxDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxDevices];

cudaError_t pool_of(int device, cudaMemPool_t *out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[device]) {
        cudaMemPoolProps pp;
        memset(&pp, 0, sizeof pp);
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &pp);
        if (e != cudaSuccess) return e;
        uint64_t keep = kPoolKeep;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        g_pools[device] = pool;
    }
    *out = g_pools[device];
    return cudaSuccess;
}

/* `bytes` of device memory from the pool, ordered on stream s */
template <class T>
cudaError_t pool_alloc(T **ptr, size_t bytes, int device, cudaStream_t s)
{
    *ptr = nullptr;
    if (bytes == 0) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = pool_of(device, &pool);
    if (e != cudaSuccess) return e;
    void *v = nullptr;
    e = cudaMallocFromPoolAsync(&v, bytes, pool, s);
    if (e == cudaSuccess) *ptr = static_cast<T *>(v);
    return e;
}

/* bytes of optical tables and geometry descriptors per launch (shared memory:
 * 227 KB per block, less 28 KB of tally columns) */
const int kMaxSharedTable = 192 * 1024;
const int64_t kMaxAttempts = 4096;       /* seeding attempts per stream before giving up */

/* seeding-generator constants for multiplier `begin` (see mc3d_rng.h) */
void make_seed_consts(uint32_t begin, mc3d_seed_consts *c)
{
    memset(c, 0, sizeof *c);
    uint64_t m = ((uint64_t)begin << 32) - 1u;
    uint64_t inv = m;
    for (int it = 0; it < 6; it++) inv *= 2u - m * inv;
    c->m = m;
    c->ninv = (uint64_t)0 - inv;
    unsigned __int128 r1 = (((unsigned __int128)1) << 64) % m;
    c->r2 = (uint64_t)((r1 * r1) % m);
    c->begin = begin;
    /* base = a^(2 16^w): one attempt is two draws of the seeding generator */
    uint64_t base = (uint64_t)(((unsigned __int128)begin * begin) % m);
    for (int w = 0; w < MC3D_JUMP_WINDOWS; w++) {
        uint64_t p = base;
        for (int d = 1; d <= 15; d++) {
            c->jump[w][d - 1] = (uint64_t)(((unsigned __int128)p * r1) % m); /* Montgomery form */
            p = (uint64_t)(((unsigned __int128)p * base) % m);
        }
        base = p; /* base^16 */
    }
}

int64_t default_streams(int64_t photons)
{
    return std::max<int64_t>(1, std::min<int64_t>(photons, MC3D_DEFAULT_STREAMS));
}

int check_table(const uint32_t *table, int64_t table_len)
{
    if (!table || table_len < 2)
        return fail(MC3D_ERR_TABLE, "safe-prime table needs at least 2 lines, got %lld",
                    (long long)table_len);
    for (int64_t i = 0; i < table_len; i++)
        if (table[i] < 2u)
            return fail(MC3D_ERR_TABLE, "safe-prime table line %lld holds multiplier %u",
                        (long long)(i + 1), table[i]);
    return MC3D_OK;
}

/* Rejected seeding attempts of one job from stream `first` on, in init_RNG's
 * sequential order (gpumcml_rng/gpumcml_rng.cu:95-114). */
int list_rejections(const mc3d_seed_consts &sc, uint64_t seed, const uint32_t *table,
                    int64_t table_len, int64_t streams, int64_t first,
                    std::vector<RejectionDev> &out)
{
    uint64_t state = mc3d_seed_jump(&sc, seed, (uint64_t)first);
    int64_t cum = 0;
    for (int64_t i = first; i < streams; i++) {
        uint32_t fora = table[1 + (i % (table_len - 1))];
        int64_t extra = 0;
        for (;;) {
            uint64_t st = mc3d_seed_attempt(state, sc.begin, fora);
            state = mc3d_mwc_next(mc3d_mwc_next(state, sc.begin), sc.begin);
            if (mc3d_seed_valid(st, fora)) break;
            if (++extra > kMaxAttempts)
                return fail(MC3D_ERR_TABLE, "multiplier %u (stream %lld) yields no valid seed",
                            fora, (long long)i);
        }
        if (extra) {
            cum += extra;
            out.push_back(RejectionDev{i, cum});
        }
    }
    return MC3D_OK;
}

/* Refractive-index classes of geometry `gi`'s tissues 0..max_tissue: two tissues
 * share a class when their index is equal in every optical set that a job uses
 * with this geometry; air (tissue 0) has a class of its own.  Returns whether two
 * tissues share one (otherwise the class map equals the tissue map). */
bool index_classes(int gi, int max_tissue, const mc3d_props *props, const mc3d_job *jobs,
                   int njobs, uint8_t classes[256])
{
    std::vector<int> sets;
    for (int j = 0; j < njobs; j++)
        if (jobs[j].geom == gi && std::find(sets.begin(), sets.end(), jobs[j].props) == sets.end())
            sets.push_back(jobs[j].props);
    for (int t = 0; t < 256; t++) classes[t] = (uint8_t)t;
    if (sets.empty()) return false;
    std::vector<std::vector<float>> keys; /* index of class c + 1 in each set */
    bool shared = false;
    for (int t = 1; t <= max_tissue; t++) {
        std::vector<float> key;
        for (int q : sets) key.push_back(props[q].n[t]);
        size_t c = 0;
        while (c < keys.size() && keys[c] != key) c++;
        if (c == keys.size()) keys.push_back(key);
        else shared = true;
        classes[t] = (uint8_t)(c + 1);
    }
    return shared;
}

} /* namespace */

/* the seeding helpers and the error text, for the other host files of the library */
namespace mc3d {
void set_last_error(const char *msg) { g_err = msg; }
void make_seed_consts_host(uint32_t begin, mc3d_seed_consts *c) { make_seed_consts(begin, c); }
int list_rejections_host(const mc3d_seed_consts &sc, uint64_t seed, const uint32_t *table,
                         int64_t table_len, int64_t streams, int64_t first,
                         std::vector<RejectionDev> &out, std::string *err)
{
    int st = list_rejections(sc, seed, table, table_len, streams, first, out);
    if (st && err) *err = g_err;
    return st;
}
} /* namespace mc3d */

struct mc3d_plan {
    int device = 0;
    int math = MC3D_MATH_FAST;
    int variant = 0; /* fast kernel variant bits (MC3D_VARIANT_*) */
    int block = 256;
    int grid = 0;
    size_t smem = 0;
    cudaStream_t stream = nullptr;
    int njobs = 0;
    std::vector<int64_t> job_bins;
    std::vector<int64_t> job_photons;
    int64_t total_bins = 0;
    int64_t total_photons = 0;
    std::vector<uint8_t *> d_grids;
    std::vector<uint16_t *> d_cells; /* packed tissue | safe distance (merged steps) */
    bool jump = false;
    JobDev *d_jobs = nullptr;
    GeomDev *d_geoms = nullptr;
    float4 *d_props = nullptr;
    uint32_t *d_mult = nullptr;
    RejectionDev *d_rej = nullptr;
    unsigned long long *d_tally = nullptr; /* drs | drs_sq | trans | totals | counter */
    unsigned long long *d_amap = nullptr;  /* absorption map, all jobs' voxels */
    std::vector<int64_t> job_voxels;
    int64_t total_voxels = 0;
    PhotonRecord *d_log = nullptr;
    mc3d_photon_record *h_log = nullptr;
    volatile int32_t *h_cancel = nullptr;
    int *d_cancel = nullptr;
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    bool cancel_registered = false;
    KernelParams P;
};

static void plan_free(mc3d_plan *p)
{
    if (!p) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(p->device);
    /* executes may be in flight on any stream: wait for the device, as cudaFree
     * would, before the buffers go back to the pool */
    cudaDeviceSynchronize();
    if (p->stream) {
        std::vector<void *> bufs(p->d_grids.begin(), p->d_grids.end());
        bufs.insert(bufs.end(), p->d_cells.begin(), p->d_cells.end());
        for (void *b : {(void *)p->d_jobs, (void *)p->d_geoms, (void *)p->d_props,
                        (void *)p->d_mult, (void *)p->d_rej, (void *)p->d_tally,
                        (void *)p->d_amap, (void *)p->d_log})
            bufs.push_back(b);
        for (void *b : bufs)
            if (b) cudaFreeAsync(b, p->stream);
        cudaStreamSynchronize(p->stream);
    }
    if (p->cancel_registered) cudaHostUnregister((void *)p->h_cancel);
    if (p->graph_exec) cudaGraphExecDestroy(p->graph_exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->stream) cudaStreamDestroy(p->stream);
    cudaSetDevice(prev);
    delete p;
}

extern "C" {

const char *mc3d_last_error(void) { return g_err.c_str(); }

int mc3d_abi_version(void) { return MC3D_ABI_VERSION; }

void mc3d_default_options(mc3d_options *opt)
{
    if (!opt) return;
    memset(opt, 0, sizeof *opt);
    opt->math = MC3D_MATH_FAST;
}

int mc3d_plan_create(mc3d_plan **plan_out, const mc3d_geom *geoms, int32_t ngeoms,
                     const mc3d_props *props, int32_t nprops, const mc3d_job *jobs,
                     int32_t njobs, const uint32_t *table, int64_t table_len,
                     const mc3d_options *opt_in)
{
    if (!plan_out) return fail(MC3D_ERR_ARG, "plan pointer is NULL");
    *plan_out = nullptr;
    if (!geoms || ngeoms <= 0 || !props || nprops <= 0 || !jobs || njobs <= 0)
        return fail(MC3D_ERR_ARG, "need at least one geometry, optical set and job");
    int st = check_table(table, table_len);
    if (st) return st;
    mc3d_options opt;
    if (opt_in) opt = *opt_in;
    else mc3d_default_options(&opt);
    if (opt.math != MC3D_MATH_FAST && opt.math != MC3D_MATH_EXACT && opt.math != MC3D_MATH_F64)
        return fail(MC3D_ERR_ARG, "unknown math mode %d", opt.math);
    if (opt.steps != MC3D_STEPS_MERGED && opt.steps != MC3D_STEPS_VOXEL)
        return fail(MC3D_ERR_ARG, "unknown step mode %d", opt.steps);
    if (opt.block < 0 || opt.block > 256 || (opt.block % 32) != 0)
        return fail(MC3D_ERR_ARG, "block must be a multiple of 32 up to 256, got %d", opt.block);

    /* ---- validate geometry and optical sets */
    std::vector<int> max_tissue(ngeoms, 0);
    for (int i = 0; i < ngeoms; i++) {
        const mc3d_geom &g = geoms[i];
        if (g.nx <= 0 || g.ny <= 0 || g.nz <= 0 || !g.tissue)
            return fail(MC3D_ERR_GEOMETRY, "geometry %d: bad size %dx%dx%d", i, g.nx, g.ny, g.nz);
        if (!(g.dx > 0) || !(g.dy > 0) || !(g.dz > 0) || !std::isfinite(g.dx) ||
            !std::isfinite(g.dy) || !std::isfinite(g.dz))
            return fail(MC3D_ERR_GEOMETRY, "geometry %d: bad voxel size", i);
        int64_t nv = (int64_t)g.nx * g.ny * g.nz;
        uint8_t mx = 0;
        for (int64_t v = 0; v < nv; v++) mx = std::max(mx, g.tissue[v]);
        max_tissue[i] = mx;
    }
    std::vector<int> props_offset(nprops);
    int entries = 0;
    for (int i = 0; i < nprops; i++) {
        const mc3d_props &p = props[i];
        if (p.num_tissue_types < 2 || p.num_tissue_types > 256 || !p.mua || !p.mus || !p.g ||
            !p.n)
            return fail(MC3D_ERR_PROPS, "optical set %d: needs 2..256 tissue types", i);
        for (int t = 0; t < p.num_tissue_types; t++)
            if (!std::isfinite(p.mua[t]) || !std::isfinite(p.mus[t]) || !std::isfinite(p.g[t]) ||
                !std::isfinite(p.n[t]))
                return fail(MC3D_ERR_PROPS, "optical set %d: tissue %d not finite", i, t);
        props_offset[i] = entries;
        entries += 3 * p.num_tissue_types;
    }
    if ((int64_t)entries * 16 + (int64_t)ngeoms * (int64_t)sizeof(GeomDev) > kMaxSharedTable)
        return fail(MC3D_ERR_CAPACITY,
                    "optical tables and geometry descriptors need %lld bytes of shared memory "
                    "(max %d)", (long long)entries * 16 + (long long)ngeoms * sizeof(GeomDev),
                    kMaxSharedTable);

    mc3d_seed_consts sc;
    make_seed_consts(table[0], &sc);

    mc3d_plan *p = new mc3d_plan();
    p->device = opt.device;
    p->math = opt.math;
    p->njobs = njobs;
    p->h_log = opt.photon_log;
    p->h_cancel = opt.cancel;
    p->use_graph = opt.use_graph != 0;

    std::vector<JobDev> jh(njobs);
    int64_t stream_base = 0, bin_base = 0, photon_base = 0, scan_base = 0, voxel_base = 0;
    for (int j = 0; j < njobs; j++) {
        const mc3d_job &jb = jobs[j];
        if (jb.geom < 0 || jb.geom >= ngeoms || jb.props < 0 || jb.props >= nprops) {
            delete p;
            return fail(MC3D_ERR_ARG, "job %d: geometry/optical index out of range", j);
        }
        if (jb.photons < 0 || jb.streams < 0 || (jb.beam != 0 && jb.beam != 1)) {
            delete p;
            return fail(MC3D_ERR_ARG, "job %d: bad photons/streams/beam", j);
        }
        if (max_tissue[jb.geom] >= props[jb.props].num_tissue_types) {
            delete p;
            return fail(MC3D_ERR_TISSUE_RANGE,
                        "job %d: geometry uses tissue type %d, optical set has %d", j,
                        max_tissue[jb.geom], props[jb.props].num_tissue_types);
        }
        if (!mc3d_user_seed_valid(jb.seed, table[0])) {
            delete p;
            return fail(MC3D_ERR_SEED, "%llu not a valid seed!", (unsigned long long)jb.seed);
        }
        int64_t S = jb.streams ? jb.streams : default_streams(jb.photons);
        int64_t first = jb.stream_first, count = jb.stream_count ? jb.stream_count : S - first;
        if (first < 0 || count < 0 || first + count > S) {
            delete p;
            return fail(MC3D_ERR_ARG, "job %d: stream range [%lld, %lld) outside %lld streams", j,
                        (long long)first, (long long)(first + count), (long long)S);
        }
        const mc3d_geom &g = geoms[jb.geom];
        JobDev &d = jh[j];
        memset(&d, 0, sizeof d);
        d.stream_base = stream_base;
        d.stream_first = first;
        d.scan_base = scan_base;
        d.streams = S;
        d.per_stream = jb.photons / S;
        d.remainder = jb.photons % S;
        d.bin_offset = bin_base;
        d.photon_base = photon_base;
        d.amap_offset = voxel_base;
        d.seed = jb.seed;
        d.geom = jb.geom;
        d.props_offset = props_offset[jb.props];
        d.beam = jb.beam;
        int64_t bins = (int64_t)g.nx * g.ny;
        int64_t voxels = bins * g.nz;
        p->job_bins.push_back(bins);
        p->job_voxels.push_back(voxels);
        voxel_base += voxels;
        p->job_photons.push_back(jb.photons);
        stream_base += count;
        d.stream_base_end = stream_base;
        scan_base += first + count;
        bin_base += bins;
        photon_base += jb.photons;
    }
    p->total_bins = bin_base;
    p->total_voxels = opt.absorption_map ? voxel_base : 0;
    p->total_photons = photon_base;

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        delete p;
        return fail(MC3D_ERR_NO_DEVICE, "no CUDA device");
    }
    if (opt.device < 0 || opt.device >= ndev) {
        delete p;
        return fail(MC3D_ERR_ARG, "device %d out of range (%d devices)", opt.device, ndev);
    }
    int prev = 0;
    cudaGetDevice(&prev);
    struct DeviceGuard {
        int prev;
        ~DeviceGuard() { cudaSetDevice(prev); }
    } guard{prev};

#define PLAN_TRY(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) {                                                              \
            plan_free(p);                                                                     \
            return fail(MC3D_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_));              \
        }                                                                                     \
    } while (0)

    PLAN_TRY(cudaSetDevice(p->device));
    PLAN_TRY(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));

    /* ---- geometry grids and descriptors */
    std::vector<GeomDev> gh(ngeoms);
    p->d_grids.assign(ngeoms, nullptr);
    p->jump = p->math != MC3D_MATH_EXACT && opt.steps != MC3D_STEPS_VOXEL;
    /* the merged kernel indexes its cell map in 32 bits: larger grids step per face */
    for (int i = 0; i < ngeoms; i++)
        if ((uint64_t)geoms[i].nx * geoms[i].ny * ((uint64_t)geoms[i].nz + MC3D_SAFE_CAP) >=
            (1ull << 32))
            p->jump = false;
    size_t max_map = 0; /* largest safe-distance map, nz + MC3D_SAFE_CAP slices */
    for (int i = 0; i < ngeoms; i++) {
        const mc3d_geom &g = geoms[i];
        size_t nv = (size_t)g.nx * g.ny * g.nz;
        max_map = std::max(max_map, (size_t)g.nx * g.ny * (g.nz + MC3D_SAFE_CAP));
        PLAN_TRY(pool_alloc(&p->d_grids[i], nv, p->device, p->stream));
        PLAN_TRY(cudaMemcpyAsync(p->d_grids[i], g.tissue, nv, cudaMemcpyHostToDevice, p->stream));
        GeomDev &d = gh[i];
        memset(&d, 0, sizeof d);
        d.nx = g.nx; d.ny = g.ny; d.nz = g.nz;
        d.dx = (float)g.dx; d.dy = (float)g.dy; d.dz = (float)g.dz;
        /* geometry->length_x = sample_dx*num_x in float (src/mc3d_io.cu:143-145) */
        d.Lx = d.dx * g.nx; d.Ly = d.dy * g.ny; d.Lz = d.dz * g.nz;
        d.rdx = 1.0f / d.dx; d.rdy = 1.0f / d.dy; d.rdz = 1.0f / d.dz;
        d.tissue = p->d_grids[i];
    }
    if (p->jump) {
        /* per geometry: the safe-distance maps of the tissue grid and of its
         * refractive-index classes, packed with the tissue into 16-bit cells
         * (scratch: two pass buffers, the two maps and the class grid) */
        p->d_cells.assign(ngeoms, nullptr);
        size_t max_vox = 0;
        for (int i = 0; i < ngeoms; i++)
            max_vox = std::max(max_vox, (size_t)geoms[i].nx * geoms[i].ny * geoms[i].nz);
        uint8_t *tmp = nullptr;
        PLAN_TRY(pool_alloc(&tmp, 4 * max_map + max_vox, p->device, p->stream));
        uint8_t *map_t = tmp + 2 * max_map, *map_n = tmp + 3 * max_map, *cls = tmp + 4 * max_map;
        cudaError_t e = cudaSuccess;
        for (int i = 0; i < ngeoms && e == cudaSuccess; i++) {
            const mc3d_geom &g = geoms[i];
            size_t nmap = (size_t)g.nx * g.ny * (g.nz + MC3D_SAFE_CAP);
            uint8_t classes[256];
            const bool shared = index_classes(i, max_tissue[i], props, jobs, njobs, classes);
            e = pool_alloc(&p->d_cells[i], 2 * nmap, p->device, p->stream);
            if (e == cudaSuccess)
                e = launch_safe_distance(p->d_grids[i], g.nx, g.ny, g.nz, map_t, tmp,
                                         tmp + max_map, p->stream);
            if (e == cudaSuccess && shared)
                e = launch_index_classes(p->d_grids[i], (int64_t)g.nx * g.ny * g.nz, classes, cls,
                                         p->stream);
            if (e == cudaSuccess && shared)
                e = launch_safe_distance(cls, g.nx, g.ny, g.nz, map_n, tmp, tmp + max_map,
                                         p->stream);
            if (e == cudaSuccess)
                e = launch_pack_cells(p->d_grids[i], map_t, shared ? map_n : map_t, g.nx, g.ny,
                                      g.nz, p->d_cells[i], p->stream);
            gh[i].cells = p->d_cells[i];
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
        cudaFreeAsync(tmp, p->stream);
        PLAN_TRY(e);
    }
    PLAN_TRY(pool_alloc(&p->d_geoms, sizeof(GeomDev) * ngeoms, p->device, p->stream));
    PLAN_TRY(cudaMemcpyAsync(p->d_geoms, gh.data(), sizeof(GeomDev) * ngeoms,
                             cudaMemcpyHostToDevice, p->stream));

    /* ---- optical tables */
    /* three float4 per tissue; every derived value is the float the reference
     * computes per step (IEEE, no contraction: this file is built with
     * -ffp-contract=off), except 1/mu_t, which only the fast kernel reads */
    std::vector<float4> tab(entries);
    for (int i = 0; i < nprops; i++)
        for (int t = 0; t < props[i].num_tissue_types; t++) {
            float mua = props[i].mua[t], mus = props[i].mus[t], g = props[i].g[t];
            volatile float mut = mua + mus;
            volatile float frac = mua / mut, rmut = 1.0f / mut, g2 = g * g, twog = 2 * g;
            volatile float inv2g = 1.0f / twog;
            float4 *e = &tab[props_offset[i] + 3 * t];
            e[0] = make_float4(mua, mus, g, props[i].n[t]);
            e[1] = make_float4(mut, frac, rmut, inv2g);
            e[2] = make_float4(1 - g2, 1 - g, twog, 1 + g2);
        }
    PLAN_TRY(pool_alloc(&p->d_props, sizeof(float4) * entries, p->device, p->stream));
    PLAN_TRY(cudaMemcpyAsync(p->d_props, tab.data(), sizeof(float4) * entries,
                             cudaMemcpyHostToDevice, p->stream));
    PLAN_TRY(pool_alloc(&p->d_mult, sizeof(uint32_t) * table_len, p->device, p->stream));
    PLAN_TRY(cudaMemcpyAsync(p->d_mult, table, sizeof(uint32_t) * table_len,
                             cudaMemcpyHostToDevice, p->stream));

    /* ---- jobs, then the seeding scan for rejected attempts */
    PLAN_TRY(pool_alloc(&p->d_jobs, sizeof(JobDev) * njobs, p->device, p->stream));
    PLAN_TRY(cudaMemcpyAsync(p->d_jobs, jh.data(), sizeof(JobDev) * njobs,
                             cudaMemcpyHostToDevice, p->stream));
    size_t tally_words = 3 * (size_t)p->total_bins + (size_t)njobs * MC3D_NUM_TOTALS + 1;
    PLAN_TRY(pool_alloc(&p->d_tally, tally_words * sizeof(unsigned long long), p->device,
                        p->stream));
    unsigned long long *first_reject = p->d_tally; /* scratch reuse before the first run */
    PLAN_TRY(cudaMemsetAsync(first_reject, 0xff, sizeof(unsigned long long) * njobs, p->stream));
    PLAN_TRY(launch_seed_scan(p->d_jobs, njobs, p->d_mult, table_len, sc, scan_base,
                              first_reject, p->stream));
    std::vector<unsigned long long> fr(njobs);
    PLAN_TRY(cudaMemcpyAsync(fr.data(), first_reject, sizeof(unsigned long long) * njobs,
                             cudaMemcpyDeviceToHost, p->stream));
    PLAN_TRY(cudaStreamSynchronize(p->stream));
    std::vector<RejectionDev> rej;
    bool any_rej = false;
    for (int j = 0; j < njobs; j++) {
        jh[j].rej_offset = (int32_t)rej.size();
        if (fr[j] != ULLONG_MAX) {
            any_rej = true;
            int s2 = list_rejections(sc, jh[j].seed, table, table_len,
                                     jh[j].stream_first + (jh[j].stream_base_end - jh[j].stream_base),
                                     (int64_t)fr[j], rej);
            if (s2) {
                std::string msg = g_err;
                plan_free(p);
                return fail(s2, "%s", msg.c_str());
            }
        }
        jh[j].rej_count = (int32_t)(rej.size() - jh[j].rej_offset);
    }
    if (rej.empty()) rej.push_back(RejectionDev{INT64_MAX, 0});
    PLAN_TRY(pool_alloc(&p->d_rej, sizeof(RejectionDev) * rej.size(), p->device, p->stream));
    PLAN_TRY(cudaMemcpyAsync(p->d_rej, rej.data(), sizeof(RejectionDev) * rej.size(),
                             cudaMemcpyHostToDevice, p->stream));
    if (any_rej)
        PLAN_TRY(cudaMemcpyAsync(p->d_jobs, jh.data(), sizeof(JobDev) * njobs,
                                 cudaMemcpyHostToDevice, p->stream));

    if (p->total_voxels)
        PLAN_TRY(pool_alloc(&p->d_amap, sizeof(unsigned long long) * p->total_voxels, p->device,
                            p->stream));
    if (p->h_log)
        PLAN_TRY(pool_alloc(&p->d_log,
                            sizeof(PhotonRecord) * std::max<int64_t>(1, p->total_photons),
                            p->device, p->stream));
    if (p->h_cancel) {
        PLAN_TRY(cudaHostRegister((void *)p->h_cancel, sizeof(int32_t), cudaHostRegisterMapped));
        p->cancel_registered = true;
        PLAN_TRY(cudaHostGetDevicePointer((void **)&p->d_cancel, (void *)p->h_cancel, 0));
    }

    /* ---- launch shape: one resident wave, all SMs */
    /* the two attributes needed, not the whole cudaDeviceProp (a slower query) */
    int num_sms = 0, smem_optin = 0;
    PLAN_TRY(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, p->device));
    PLAN_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                    p->device));
    p->block = opt.block ? opt.block : 256;
    p->smem = sizeof(float4) * entries + sizeof(GeomDev) * ngeoms;
    /* The kernels' static shared memory (28 KB of per-thread tallies) counts
     * against the 48 KB a block gets without opting in, so the kernels always opt
     * in, to the device's whole per-block limit: the attribute is per function,
     * and a lower value would break a live plan that needs more. */
    {
        cudaFuncAttributes fa;
        PLAN_TRY(p->math == MC3D_MATH_FAST    ? attributes_photon_fast(&fa)
                 : p->math == MC3D_MATH_EXACT ? attributes_photon_exact(&fa)
                                              : attributes_photon_f64(&fa));
        const size_t max_dyn = (size_t)smem_optin - fa.sharedSizeBytes;
        if (p->smem > max_dyn) {
            plan_free(p);
            return fail(MC3D_ERR_CAPACITY, "optical tables and geometry descriptors need %zu B "
                        "of shared memory, the device allows %zu", p->smem, max_dyn);
        }
        PLAN_TRY(p->math == MC3D_MATH_FAST    ? smem_limit_photon_fast(max_dyn)
                 : p->math == MC3D_MATH_EXACT ? smem_limit_photon_exact(max_dyn)
                                              : smem_limit_photon_f64(max_dyn));
    }
    p->variant = (p->jump ? 0 : MC3D_VARIANT_VOXEL_STEPS) | (ngeoms == 1 ? MC3D_VARIANT_ONE_GEOM : 0);
    int bps = 0;
    PLAN_TRY(p->math == MC3D_MATH_FAST ? occupancy_photon_fast(p->block, p->smem, &bps, p->variant)
             : p->math == MC3D_MATH_EXACT ? occupancy_photon_exact(p->block, p->smem, &bps)
                                          : occupancy_photon_f64(p->block, p->smem, &bps, p->variant));
    if (bps <= 0) {
        plan_free(p);
        return fail(MC3D_ERR_CAPACITY, "kernel does not fit an SM with block %d", opt.block);
    }
    if (opt.blocks_per_sm > 0) bps = std::min(bps, (int)opt.blocks_per_sm);
    p->grid = num_sms * bps;

    KernelParams &P = p->P;
    memset(&P, 0, sizeof P);
    P.jobs = p->d_jobs;
    P.geoms = p->d_geoms;
    P.geom0 = gh[0];
    P.props_table = p->d_props;
    P.multipliers = p->d_mult;
    P.rejections = p->d_rej;
    P.drs = p->d_tally;
    P.drs_sq = p->d_tally + p->total_bins;
    P.trans = p->d_tally + 2 * p->total_bins;
    P.totals = p->d_tally + 3 * p->total_bins;
    P.work_counter = p->d_tally + 3 * p->total_bins + (size_t)njobs * MC3D_NUM_TOTALS;
    P.cancel = p->d_cancel;
    P.photon_log = p->d_log;
    P.amap = p->d_amap;
    P.num_multipliers = table_len;
    P.mult_magic = UINT64_MAX / (uint64_t)(table_len - 1);
    P.total_streams = stream_base;
    P.max_steps = opt.max_steps > 0 ? std::min<int64_t>(opt.max_steps, INT32_MAX) : (1 << 24);
    P.njobs = njobs;
    P.ngeoms = ngeoms;
    P.props_entries = entries;
    P.seed = sc;
    PLAN_TRY(cudaStreamSynchronize(p->stream));
    *plan_out = p;
    return MC3D_OK;
#undef PLAN_TRY
}

/* clear the tallies and launch: the work of one execute, on stream s */
static int plan_enqueue(mc3d_plan *p, cudaStream_t s)
{
    size_t tally_words = 3 * (size_t)p->total_bins + (size_t)p->njobs * MC3D_NUM_TOTALS + 1;
    CUDA_TRY(cudaMemsetAsync(p->d_tally, 0, tally_words * sizeof(unsigned long long), s));
    if (p->d_amap)
        CUDA_TRY(cudaMemsetAsync(p->d_amap, 0, sizeof(unsigned long long) * p->total_voxels, s));
    if (p->math == MC3D_MATH_FAST)
        CUDA_TRY(launch_photon_fast(p->P, p->grid, p->block, p->smem, s, p->variant));
    else if (p->math == MC3D_MATH_EXACT)
        CUDA_TRY(launch_photon_exact(p->P, p->grid, p->block, p->smem, s));
    else CUDA_TRY(launch_photon_f64(p->P, p->grid, p->block, p->smem, s, p->variant));
    return MC3D_OK;
}

int mc3d_plan_execute(mc3d_plan *p, void *stream)
{
    if (!p) return fail(MC3D_ERR_ARG, "plan is NULL");
    cudaStream_t s = stream ? (cudaStream_t)stream : p->stream;
    CUDA_TRY(cudaSetDevice(p->device));
    if (!p->use_graph) return plan_enqueue(p, s);
    if (!p->graph_exec) {
        /* capture on the plan's own stream, then replay on any stream */
        CUDA_TRY(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
        int st = plan_enqueue(p, p->stream);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(p->stream, &g);
        if (st) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        p->graph = g;
        CUDA_TRY(cudaGraphInstantiate(&p->graph_exec, p->graph, 0));
    }
    CUDA_TRY(cudaGraphLaunch(p->graph_exec, s));
    return MC3D_OK;
}

int mc3d_plan_read(mc3d_plan *p, mc3d_out *out)
{
    if (!p || !out) return fail(MC3D_ERR_ARG, "plan or out is NULL");
    CUDA_TRY(cudaSetDevice(p->device));
    CUDA_TRY(cudaDeviceSynchronize());
    std::vector<unsigned long long> tot((size_t)p->njobs * MC3D_NUM_TOTALS);
    CUDA_TRY(cudaMemcpy(tot.data(), p->P.totals, tot.size() * sizeof(unsigned long long),
                        cudaMemcpyDeviceToHost));
    int64_t off = 0, voff = 0;
    for (int j = 0; j < p->njobs; j++) {
        if (out[j].absorption) {
            if (!p->d_amap) return fail(MC3D_ERR_ARG, "absorption map not enabled in the plan");
            CUDA_TRY(cudaMemcpy(out[j].absorption, p->d_amap + voff,
                                sizeof(uint64_t) * p->job_voxels[j], cudaMemcpyDeviceToHost));
        }
        voff += p->job_voxels[j];
        size_t nb = (size_t)p->job_bins[j] * sizeof(uint64_t);
        if (out[j].drs) CUDA_TRY(cudaMemcpy(out[j].drs, p->P.drs + off, nb, cudaMemcpyDeviceToHost));
        if (out[j].drs_sq)
            CUDA_TRY(cudaMemcpy(out[j].drs_sq, p->P.drs_sq + off, nb, cudaMemcpyDeviceToHost));
        if (out[j].trans)
            CUDA_TRY(cudaMemcpy(out[j].trans, p->P.trans + off, nb, cudaMemcpyDeviceToHost));
        memcpy(&out[j].totals, tot.data() + (size_t)j * MC3D_NUM_TOTALS, sizeof(mc3d_totals));
        off += p->job_bins[j];
    }
    if (p->h_log && p->d_log && p->total_photons > 0)
        CUDA_TRY(cudaMemcpy(p->h_log, p->d_log, sizeof(PhotonRecord) * p->total_photons,
                            cudaMemcpyDeviceToHost));
    if (p->h_cancel && *p->h_cancel)
        return fail(MC3D_ERR_CANCELLED, "cancelled; results cover the photons finished so far");
    return MC3D_OK;
}

int mc3d_plan_shape(const mc3d_plan *p, int32_t *block, int32_t *grid, int32_t *smem)
{
    if (!p) return fail(MC3D_ERR_ARG, "plan is NULL");
    if (block) *block = p->block;
    if (grid) *grid = p->grid;
    if (smem) *smem = (int32_t)p->smem;
    return MC3D_OK;
}

int mc3d_plan_device_totals(const mc3d_plan *p, void **ptr)
{
    if (!p || !ptr) return fail(MC3D_ERR_ARG, "plan or ptr is NULL");
    *ptr = (void *)p->P.totals;
    return MC3D_OK;
}

void mc3d_plan_destroy(mc3d_plan *p) { plan_free(p); }

int mc3d_run(const mc3d_geom *geoms, int32_t ngeoms, const mc3d_props *props, int32_t nprops,
             const mc3d_job *jobs, int32_t njobs, const uint32_t *table, int64_t table_len,
             const mc3d_options *opt, mc3d_out *out)
{
    if (!out) return fail(MC3D_ERR_ARG, "out is NULL");
    mc3d_plan *p = nullptr;
    int st = mc3d_plan_create(&p, geoms, ngeoms, props, nprops, jobs, njobs, table, table_len, opt);
    if (st) return st;
    st = mc3d_plan_execute(p, nullptr);
    if (!st) st = mc3d_plan_read(p, out);
    std::string keep = g_err;
    plan_free(p);
    g_err = keep;
    return st;
}

int mc3d_stream_seeds(const mc3d_job *job, const uint32_t *table, int64_t table_len,
                      int64_t first, int64_t count, uint64_t *x_out, uint32_t *a_out,
                      int32_t device)
{
    if (!job || !x_out || !a_out || first < 0 || count < 0)
        return fail(MC3D_ERR_ARG, "bad arguments");
    int st = check_table(table, table_len);
    if (st) return st;
    if (!mc3d_user_seed_valid(job->seed, table[0]))
        return fail(MC3D_ERR_SEED, "%llu not a valid seed!", (unsigned long long)job->seed);
    int64_t S = job->streams ? job->streams : default_streams(job->photons);
    if (first + count > S) return fail(MC3D_ERR_ARG, "streams beyond the job's %lld", (long long)S);
    if (count == 0) return MC3D_OK;
    mc3d_seed_consts sc;
    make_seed_consts(table[0], &sc);
    /* rejections are found on the host here: the ranges asked for are small */
    std::vector<RejectionDev> rej;
    st = list_rejections(sc, job->seed, table, table_len, first + count, 0, rej);
    if (st) return st;
    JobDev jd;
    memset(&jd, 0, sizeof jd);
    jd.streams = S;
    jd.seed = job->seed;
    jd.rej_offset = 0;
    jd.rej_count = (int32_t)rej.size();
    if (rej.empty()) rej.push_back(RejectionDev{INT64_MAX, 0});

    CUDA_TRY(cudaSetDevice(device));
    JobDev *d_job = nullptr;
    uint32_t *d_mult = nullptr;
    RejectionDev *d_rej = nullptr;
    uint64_t *d_x = nullptr;
    uint32_t *d_a = nullptr;
    cudaError_t e = cudaSuccess;
    do {
        if ((e = cudaMalloc(&d_job, sizeof jd)) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_mult, sizeof(uint32_t) * table_len)) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_rej, sizeof(RejectionDev) * rej.size())) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_x, sizeof(uint64_t) * count)) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_a, sizeof(uint32_t) * count)) != cudaSuccess) break;
        if ((e = cudaMemcpy(d_job, &jd, sizeof jd, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = cudaMemcpy(d_mult, table, sizeof(uint32_t) * table_len, cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            break;
        if ((e = cudaMemcpy(d_rej, rej.data(), sizeof(RejectionDev) * rej.size(),
                            cudaMemcpyHostToDevice)) != cudaSuccess)
            break;
        KernelParams P;
        memset(&P, 0, sizeof P);
        P.jobs = d_job;
        P.multipliers = d_mult;
        P.num_multipliers = table_len;
        P.mult_magic = UINT64_MAX / (uint64_t)(table_len - 1);
        P.rejections = d_rej;
        P.njobs = 1;
        P.seed = sc;
        if ((e = launch_seed_dump(P, first, count, d_x, d_a, nullptr)) != cudaSuccess) break;
        if ((e = cudaMemcpy(x_out, d_x, sizeof(uint64_t) * count, cudaMemcpyDeviceToHost)) !=
            cudaSuccess)
            break;
        e = cudaMemcpy(a_out, d_a, sizeof(uint32_t) * count, cudaMemcpyDeviceToHost);
    } while (0);
    cudaFree(d_job);
    cudaFree(d_mult);
    cudaFree(d_rej);
    cudaFree(d_x);
    cudaFree(d_a);
    if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, "stream seeds: %s", cudaGetErrorString(e));
    return MC3D_OK;
}

int mc3d_mwc_draws(const uint64_t *x, const uint32_t *a, int64_t ngen, int64_t n, float *out,
                   int32_t device)
{
    if (!x || !a || !out || ngen < 0 || n < 0) return fail(MC3D_ERR_ARG, "bad arguments");
    if (ngen == 0 || n == 0) return MC3D_OK;
    CUDA_TRY(cudaSetDevice(device));
    uint64_t *d_x = nullptr;
    uint32_t *d_a = nullptr;
    float *d_o = nullptr;
    cudaError_t e = cudaSuccess;
    do {
        if ((e = cudaMalloc(&d_x, sizeof(uint64_t) * ngen)) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_a, sizeof(uint32_t) * ngen)) != cudaSuccess) break;
        if ((e = cudaMalloc(&d_o, sizeof(float) * ngen * n)) != cudaSuccess) break;
        if ((e = cudaMemcpy(d_x, x, sizeof(uint64_t) * ngen, cudaMemcpyHostToDevice)) != cudaSuccess)
            break;
        if ((e = cudaMemcpy(d_a, a, sizeof(uint32_t) * ngen, cudaMemcpyHostToDevice)) != cudaSuccess)
            break;
        if ((e = launch_mwc_draws(d_x, d_a, ngen, n, d_o, nullptr)) != cudaSuccess) break;
        e = cudaMemcpy(out, d_o, sizeof(float) * ngen * n, cudaMemcpyDeviceToHost);
    } while (0);
    cudaFree(d_x);
    cudaFree(d_a);
    cudaFree(d_o);
    if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, "mwc draws: %s", cudaGetErrorString(e));
    return MC3D_OK;
}

int mc3d_safe_distance(const uint8_t *tissue, int32_t nx, int32_t ny, int32_t nz,
                       uint8_t *radius, int32_t device)
{
    if (!tissue || !radius || nx <= 0 || ny <= 0 || nz <= 0)
        return fail(MC3D_ERR_ARG, "bad arguments");
    CUDA_TRY(cudaSetDevice(device));
    const size_t nv = (size_t)nx * ny * nz;
    const size_t nm = (size_t)nx * ny * (nz + MC3D_SAFE_CAP);
    uint8_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, nv + 3 * nm); /* grid | map | two scratch maps */
    if (e == cudaSuccess) e = cudaMemcpy(d, tissue, nv, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = launch_safe_distance(d, nx, ny, nz, d + nv, d + nv + nm, d + nv + 2 * nm, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(radius, d + nv, nm, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return fail(MC3D_ERR_CUDA, "safe distance: %s", cudaGetErrorString(e));
    return MC3D_OK;
}

int mc3d_run_3dmc_gpu(mc3d_ref_geometry geometry, mc3d_ref_opticalprops optProps, int num_photons,
                      double *R, double *R_tot, double *T, double *T_tot, float *A,
                      int *num_finished_photons)
{
    (void)A; /* the reference only round-trips A (src/mc3d_gpu.cu:426-427, 586) */
    if (!geometry.tissue_type || !optProps.n || !optProps.mua || !optProps.mus || !optProps.g)
        return fail(MC3D_ERR_ARG, "null geometry or optical arrays");
    int64_t nv = (int64_t)geometry.num_x * geometry.num_y * geometry.num_z;
    if (nv <= 0) return fail(MC3D_ERR_GEOMETRY, "empty geometry");
    std::vector<uint8_t> grid((size_t)nv);
    for (int64_t v = 0; v < nv; v++) {
        int t = geometry.tissue_type[v];
        if (t < 0 || t > 255) return fail(MC3D_ERR_TISSUE_RANGE, "voxel %lld has tissue %d", (long long)v, t);
        grid[v] = (uint8_t)t;
    }
    mc3d_geom g;
    memset(&g, 0, sizeof g);
    g.nx = geometry.num_x; g.ny = geometry.num_y; g.nz = geometry.num_z;
    g.dx = geometry.sample_dx; g.dy = geometry.sample_dy; g.dz = geometry.sample_dz;
    g.tissue = grid.data();
    mc3d_props pr;
    memset(&pr, 0, sizeof pr);
    pr.num_tissue_types = optProps.num_tissue_types;
    pr.mua = optProps.mua; pr.mus = optProps.mus; pr.g = optProps.g; pr.n = optProps.n;

    /* rng_init reads ./safeprimes_base32.txt (src/mc3d_rng.cu:16) */
    std::vector<uint32_t> table(1 + 230400);
    int64_t nread = 0;
    if (mc3d_safeprimes_read("safeprimes_base32.txt", table.data(), (int64_t)table.size(), &nread) ||
        nread < 2) {
        fprintf(stderr, "Couldn't find safeprimes_base32.txt.\n");
        return fail(MC3D_ERR_TABLE, "Couldn't find safeprimes_base32.txt.");
    }
    const char *env = getenv("MC3D_SEED");
    uint64_t seed = env ? strtoull(env, nullptr, 10) : (uint64_t)time(NULL);
    fprintf(stderr, "seed: %llu\n", (unsigned long long)seed);
    mc3d_job job;
    memset(&job, 0, sizeof job);
    job.photons = num_photons;
    job.seed = seed;
    job.beam = MC3D_BEAM_UNIFORM;
    int64_t nb = (int64_t)g.nx * g.ny;
    std::vector<uint64_t> drs((size_t)nb), trans((size_t)nb);
    mc3d_out out;
    memset(&out, 0, sizeof out);
    out.drs = drs.data();
    out.trans = trans.data();
    int st = mc3d_run(&g, 1, &pr, 1, &job, 1, table.data(), nread, nullptr, &out);
    if (st) return st;
    const double q = 1.0 / MC3D_WEIGHT_SCALE;
    for (int64_t b = 0; b < nb; b++) {
        if (R) R[b] += (double)drs[b] * q;
        if (T) T[b] += (double)trans[b] * q;
    }
    if (R_tot) *R_tot += (double)(out.totals.r_in + out.totals.r_out) * q;
    if (T_tot) *T_tot += (double)(out.totals.t_in + out.totals.t_out) * q;
    if (num_finished_photons) *num_finished_photons = (int)out.totals.photons;
    return MC3D_OK;
}

} /* extern "C" */
