/*
 * gpu_mc.cpp -- the `gpu-mc geometry.bin optprops.bid <params> outname` command
 * (src/mc3d_main.cu:15-98) on top of libmc3d.so.
 *
 * Same inputs, same stdout/stderr lines and the same outname_drs.bin and
 * outname_simparam.dat.  The third argument, ignored by the reference
 * (README.md:38), is read as an optional key=value file:
 *   photons=30000000  seed=<time>  beam=uniform|pencil  streams=0  math=fast|exact|f64
 *   safeprimes=safeprimes_base32.txt  max_steps=0  device=0  abs_map=0  save_trans=0
 *   steps=merged|voxel (fast math: merged crossings in uniform tissue, or one step
 *   per voxel face like the reference)
 * An unreadable file (such as the README's "dummy_argument") keeps the defaults.
 * Differences: Total diffuse reflectance is the real total (the reference never
 * accumulates R_tot), and outname_report.json records the integer tallies.
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "mc3d.h"

namespace {

struct Params {
    long long photons = 30000000; /* src/mc3d_main.cu:57 */
    unsigned long long seed = 0;
    bool seed_set = false;
    int beam = MC3D_BEAM_UNIFORM;
    long long streams = 0;
    int math = MC3D_MATH_FAST;
    int steps = MC3D_STEPS_MERGED;
    std::string safeprimes = "safeprimes_base32.txt";
    long long max_steps = 0;
    int device = 0;
    bool abs_map = false;    /* write outname_abs.bin and outname_flu.bin */
    bool save_trans = false; /* write outname_trans.bin */
};

std::string trim(const std::string &s)
{
    size_t b = s.find_first_not_of(" \t\r\n"), e = s.find_last_not_of(" \t\r\n");
    return b == std::string::npos ? "" : s.substr(b, e - b + 1);
}

bool read_params(const char *path, Params &p)
{
    std::ifstream in(path);
    if (!in) return false;
    std::string line;
    while (std::getline(in, line)) {
        size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        std::string k = trim(line.substr(0, eq)), v = trim(line.substr(eq + 1));
        if (k == "photons") p.photons = std::llround(std::stod(v));
        else if (k == "seed") { p.seed = std::stoull(v); p.seed_set = true; }
        else if (k == "beam") p.beam = (v == "pencil") ? MC3D_BEAM_PENCIL : MC3D_BEAM_UNIFORM;
        else if (k == "streams") p.streams = std::stoll(v);
        else if (k == "math")
            p.math = (v == "exact") ? MC3D_MATH_EXACT : (v == "f64") ? MC3D_MATH_F64 : MC3D_MATH_FAST;
        else if (k == "steps") p.steps = (v == "voxel") ? MC3D_STEPS_VOXEL : MC3D_STEPS_MERGED;
        else if (k == "safeprimes") p.safeprimes = v;
        else if (k == "max_steps") p.max_steps = std::stoll(v);
        else if (k == "device") p.device = std::stoi(v);
        else if (k == "abs_map") p.abs_map = std::stoi(v) != 0;
        else if (k == "save_trans") p.save_trans = std::stoi(v) != 0;
    }
    return true;
}

} /* namespace */

int main(int argc, char *argv[])
{
    if (argc < 5) {
        fprintf(stderr, "\nUsage: %s geometry.bin tissue.bid definition.txt OutputName\n", argv[0]);
        return 1;
    }
    const char *geomPath = argv[1], *tissuePath = argv[2], *defPath = argv[3], *outName = argv[4];

    int32_t nx, ny, nz;
    double dx, dy, dz;
    int st = mc3d_read_geometry_header(geomPath, &nx, &ny, &nz, &dx, &dy, &dz);
    std::vector<uint8_t> grid;
    if (st == MC3D_OK) {
        grid.resize((size_t)nx * ny * nz);
        st = mc3d_read_geometry(geomPath, grid.data(), (int64_t)grid.size());
    }
    if (st == MC3D_ERR_IO) fprintf(stderr, "The file %s was not opened\n", geomPath);
    else if (st) fprintf(stderr, "Could not read geometry %s (status %d)\n", geomPath, st);
    int32_t ntypes = 0;
    int st2 = mc3d_read_optprops(tissuePath, &ntypes, nullptr, nullptr, nullptr, nullptr, 0);
    std::vector<float> mua, mus, g, n;
    if (st2 == MC3D_OK) {
        mua.resize(ntypes); mus.resize(ntypes); g.resize(ntypes); n.resize(ntypes);
        st2 = mc3d_read_optprops(tissuePath, &ntypes, mua.data(), mus.data(), g.data(), n.data(),
                                 ntypes);
    }
    if (st2 == MC3D_ERR_IO) fprintf(stderr, "The file %s was not opened\n", tissuePath);
    else if (st2) fprintf(stderr, "Could not read optical properties %s (status %d)\n", tissuePath, st2);
    if (st != 0 || st2 != 0) return 1;
    fprintf(stderr, "\nRead geometry: %s and tissue definition: %s.\n", geomPath, tissuePath);

    std::cout << "#mua (mm-1), mus (mm-1), g, n. Rows: tissue type 1, tissue type 2, ..." << std::endl;
    for (int i = 1; i < ntypes; i++)
        std::cout << mua[i] << " " << mus[i] << " " << g[i] << " " << n[i] << std::endl;

    Params prm;
    read_params(defPath, prm);
    if (!prm.seed_set) prm.seed = (unsigned long long)time(NULL);

    std::vector<uint32_t> table((size_t)1 << 20);
    int64_t nread = 0;
    if (mc3d_safeprimes_read(prm.safeprimes.c_str(), table.data(), (int64_t)table.size(), &nread) ||
        nread < 2) {
        fprintf(stderr, "Couldn't find %s.\n", prm.safeprimes.c_str());
        return 1;
    }
    table.resize((size_t)nread);
    std::cerr << "seed: " << prm.seed << std::endl;
    fprintf(stderr, "\nPerforming MC3D simulation using CUDA.\n");

    mc3d_geom geom;
    memset(&geom, 0, sizeof geom);
    geom.nx = nx; geom.ny = ny; geom.nz = nz;
    geom.dx = dx; geom.dy = dy; geom.dz = dz;
    geom.tissue = grid.data();
    mc3d_props props;
    memset(&props, 0, sizeof props);
    props.num_tissue_types = ntypes;
    props.mua = mua.data(); props.mus = mus.data(); props.g = g.data(); props.n = n.data();
    mc3d_job job;
    memset(&job, 0, sizeof job);
    job.photons = prm.photons;
    job.streams = prm.streams;
    job.seed = prm.seed;
    job.beam = prm.beam;
    mc3d_options opt;
    mc3d_default_options(&opt);
    opt.device = prm.device;
    opt.math = prm.math;
    opt.steps = prm.steps;
    opt.max_steps = prm.max_steps;
    opt.absorption_map = prm.abs_map ? 1 : 0;

    size_t nb = (size_t)nx * ny;
    std::vector<uint64_t> drs(nb), drs_sq(nb), trans(nb);
    mc3d_out out;
    memset(&out, 0, sizeof out);
    out.drs = drs.data(); out.drs_sq = drs_sq.data(); out.trans = trans.data();
    std::vector<uint64_t> amap(prm.abs_map ? grid.size() : 0);
    if (prm.abs_map) out.absorption = amap.data();
    auto t0 = std::chrono::steady_clock::now();
    st = mc3d_run(&geom, 1, &props, 1, &job, 1, table.data(), (int64_t)table.size(), &opt, &out);
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (st) {
        fprintf(stderr, "mc3d_run failed (%d): %s\n", st, mc3d_last_error());
        return 1;
    }
    const double q = 1.0 / MC3D_WEIGHT_SCALE;
    std::vector<double> R(nb);
    for (size_t b = 0; b < nb; b++) R[b] = (double)drs[b] * q;
    long long finished = (long long)out.totals.photons;
    double totDiffR = (double)(out.totals.r_in + out.totals.r_out) * q;

    fprintf(stderr, "Total diffuse reflectance is %f.\n", totDiffR / finished);
    float geomDiffR = 0; /* float accumulation as in src/mc3d_main.cu:66-69 */
    for (size_t b = 0; b < nb; b++) geomDiffR += R[b];
    fprintf(stderr, "(diffuse reflectance over geometry area is %f)\n", geomDiffR / finished);
    fprintf(stderr, "Absorbed fraction in geometry is %f.\n", 0.0);
    fprintf(stderr, "Absorbed fraction outside geometry is NOT CALCULATED.\n");
    fprintf(stderr, "Absorbed fraction (all depths) is %f.\n",
            (double)out.totals.absorbed * q / finished);
    fprintf(stderr, "%lld photons, %llu steps in %.3f s (%.4g photons/s)\n", finished,
            (unsigned long long)out.totals.steps, secs, finished / secs);

    st = mc3d_save_diff_refl(outName, nx, ny, (float)dx, (float)dy, R.data(), finished);
    if (st) {
        fprintf(stderr, "The file was not saved.\n");
        return 1;
    }
    if (prm.save_trans) {
        std::vector<double> Tn(nb);
        for (size_t b = 0; b < nb; b++) Tn[b] = (double)trans[b] * q / finished;
        mc3d_save_property((std::string(outName) + "_trans.bin").c_str(), 2, nx, ny, 1, (float)dx,
                           (float)dy, 0.0, Tn.data());
    }
    if (prm.abs_map) {
        /* save_abs_map (src/mc3d_io.cu:229-255, never called by the reference): absorbed
         * weight per voxel per photon, and fluence = absorbed / mua of the voxel's
         * tissue.  The reference multiplies by the photon count; dividing is what
         * makes the map a fraction.  Voxels of mua = 0 get fluence 0, not inf. */
        std::vector<double> A(grid.size()), F(grid.size());
        for (size_t v = 0; v < grid.size(); v++) {
            A[v] = (double)amap[v] * q / finished;
            float m = mua[grid[v]];
            F[v] = m > 0 ? A[v] / m : 0.0;
        }
        mc3d_save_property((std::string(outName) + "_abs.bin").c_str(), 3, nx, ny, nz, (float)dx,
                           (float)dy, (float)dz, A.data());
        mc3d_save_property((std::string(outName) + "_flu.bin").c_str(), 3, nx, ny, nz, (float)dx,
                           (float)dy, (float)dz, F.data());
    }
    FILE *numPhotFile = fopen((std::string(outName) + "_simparam.dat").c_str(), "w");
    if (numPhotFile) {
        fprintf(numPhotFile, "%lld #num_photons\n", finished);
        fclose(numPhotFile);
    }
    FILE *rep = fopen((std::string(outName) + "_report.json").c_str(), "w");
    if (rep) {
        const mc3d_totals &t = out.totals;
        fprintf(rep,
                "{\"photons\": %llu, \"steps\": %llu, \"seconds\": %.6f, \"photons_per_s\": %.6g, "
                "\"seed\": %llu, \"weight_scale\": 4294967296, \"w_launched\": %llu, "
                "\"r_in\": %llu, \"r_out\": %llu, \"t_in\": %llu, \"t_out\": %llu, "
                "\"absorbed\": %llu, \"rr_killed\": %llu, \"rr_created\": %llu, \"lost\": %llu, "
                "\"capped\": %llu, \"quickfix\": %llu, \"fresnel\": %llu}\n",
                (unsigned long long)t.photons, (unsigned long long)t.steps, secs, finished / secs,
                prm.seed, (unsigned long long)t.w_launched, (unsigned long long)t.r_in,
                (unsigned long long)t.r_out, (unsigned long long)t.t_in,
                (unsigned long long)t.t_out, (unsigned long long)t.absorbed,
                (unsigned long long)t.rr_killed, (unsigned long long)t.rr_created,
                (unsigned long long)t.lost, (unsigned long long)t.capped,
                (unsigned long long)t.quickfix, (unsigned long long)t.fresnel);
        fclose(rep);
    }
    return 0;
}
