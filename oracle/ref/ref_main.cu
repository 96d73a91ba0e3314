/*
 * ref_main.cu -- driver for the reference's own run_3dmc_gpu.
 *
 * TEST INFRASTRUCTURE ONLY.  Links the reference's src/mc3d_gpu.cu,
 * src/mc3d_photons.cu and src/mc3d_io.cu, compiled unmodified where they lie,
 * and replaces only src/mc3d_main.cu so that the photon count and the seed can
 * be chosen (the reference hard-codes 30,000,000 photons at src/mc3d_main.cu:57
 * and seeds from time(NULL) at src/mc3d_gpu.cu:454; the latter is routed here by
 * compiling mc3d_gpu.cu with -Dtime=mc3d_ref_seed_clock).
 *
 *   gpu-mc-ref geometry.bin optprops.bid photons seed outname [table_dir]
 *
 * Writes outname_drs.bin through the reference's save_diff_refl, and
 * outname_ref.bin: int64 finished, double seconds, int32 nx, ny, double R[ny][nx],
 * double T[ny][nx] (un-normalised weight sums as run_3dmc_gpu leaves them).
 */
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <string>
#include <unistd.h>

#include "mc3d_gpu.h"
#include "mc3d_io.h"
#include "mc3d_types.h"

static unsigned long long g_seed = 1;

extern "C" time_t mc3d_ref_seed_clock(time_t *t)
{
    if (t) *t = (time_t)g_seed;
    return (time_t)g_seed;
}

int main(int argc, char *argv[])
{
    if (argc < 6) {
        fprintf(stderr, "usage: %s geometry.bin optprops.bid photons seed outname [table_dir]\n",
                argv[0]);
        return 2;
    }
    char geom_path[PATH_MAX], prop_path[PATH_MAX];
    if (!realpath(argv[1], geom_path) || !realpath(argv[2], prop_path)) {
        fprintf(stderr, "input file not found\n");
        return 2;
    }
    int num_photons = atoi(argv[3]);
    g_seed = strtoull(argv[4], nullptr, 10);
    std::string out = argv[5];
    if (out[0] != '/') {
        char cwd[PATH_MAX];
        if (getcwd(cwd, sizeof cwd)) out = std::string(cwd) + "/" + out;
    }
    geometry_t geometry;
    opticalprops_t optProps;
    int stat = geometry_read_from_file(&geometry, geom_path);
    stat += opticalprops_read_from_file(&optProps, prop_path);
    if (stat != 0) return 1;
    if (argc > 6 && chdir(argv[6]) != 0) {
        fprintf(stderr, "cannot enter %s\n", argv[6]);
        return 2;
    }
    size_t nb = (size_t)geometry.num_x * geometry.num_y;
    double *R = new double[nb]();
    double *T = new double[nb]();
    float *A = new float[(size_t)geometry.num_x * geometry.num_y * geometry.num_z]();
    double totR = 0, totT = 0;
    int finished = 0;
    auto t0 = std::chrono::steady_clock::now();
    run_3dmc_gpu(geometry, optProps, num_photons, R, &totR, T, &totT, A, &finished);
    cudaDeviceSynchronize();
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    save_diff_refl(geometry, R, finished, (char *)out.c_str());
    FILE *f = fopen((out + "_ref.bin").c_str(), "wb");
    if (!f) return 1;
    long long fin = finished;
    int nx = geometry.num_x, ny = geometry.num_y;
    fwrite(&fin, sizeof fin, 1, f);
    fwrite(&secs, sizeof secs, 1, f);
    fwrite(&nx, sizeof nx, 1, f);
    fwrite(&ny, sizeof ny, 1, f);
    fwrite(R, sizeof(double), nb, f);
    fwrite(T, sizeof(double), nb, f);
    fclose(f);
    fprintf(stderr, "reference: %d photons finished in %.3f s\n", finished, secs);
    return 0;
}
