/*
 * mc3d_io.cpp -- the reference's file formats (src/mc3d_io.cu:16-255), with the
 * checks the reference leaves out: a missing file returns MC3D_ERR_IO (the
 * reference calls fclose(NULL) first, :20-23, :111-114), a short file returns
 * MC3D_ERR_FORMAT (the reference ignores fread counts), and tissue indices that do
 * not fit the engine's uint8 grid return MC3D_ERR_TISSUE_RANGE.
 */
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mc3d.h"

namespace {

struct File {
    FILE *f;
    explicit File(FILE *f_) : f(f_) {}
    ~File()
    {
        if (f) fclose(f);
    }
};

int read_header(FILE *f, int32_t *nx, int32_t *ny, int32_t *nz, double *dx, double *dy,
                double *dz)
{
    int32_t dim = 0, n[3];
    double d[3];
    if (fread(&dim, sizeof dim, 1, f) != 1) return MC3D_ERR_FORMAT;
    if (dim != 3) return MC3D_ERR_FORMAT; /* "Binary is not 3D." (:121-125) */
    if (fread(n, sizeof(int32_t), 3, f) != 3) return MC3D_ERR_FORMAT;
    if (fread(d, sizeof(double), 3, f) != 3) return MC3D_ERR_FORMAT;
    if (n[0] <= 0 || n[1] <= 0 || n[2] <= 0) return MC3D_ERR_GEOMETRY;
    *nx = n[0]; *ny = n[1]; *nz = n[2];
    *dx = d[0]; *dy = d[1]; *dz = d[2];
    return MC3D_OK;
}

} /* namespace */

extern "C" {

int mc3d_read_geometry_header(const char *path, int32_t *nx, int32_t *ny, int32_t *nz,
                              double *dx, double *dy, double *dz)
{
    if (!path || !nx || !ny || !nz || !dx || !dy || !dz) return MC3D_ERR_ARG;
    File f(fopen(path, "rb"));
    if (!f.f) return MC3D_ERR_IO;
    return read_header(f.f, nx, ny, nz, dx, dy, dz);
}

int mc3d_read_geometry(const char *path, uint8_t *tissue, int64_t cap)
{
    if (!path || !tissue) return MC3D_ERR_ARG;
    File f(fopen(path, "rb"));
    if (!f.f) return MC3D_ERR_IO;
    int32_t nx, ny, nz;
    double dx, dy, dz;
    int st = read_header(f.f, &nx, &ny, &nz, &dx, &dy, &dz);
    if (st) return st;
    int64_t nv = (int64_t)nx * ny * nz;
    if (nv > cap) return MC3D_ERR_ARG;
    std::vector<int32_t> row((size_t)nx);
    for (int64_t r = 0; r < (int64_t)ny * nz; r++) {
        if (fread(row.data(), sizeof(int32_t), (size_t)nx, f.f) != (size_t)nx)
            return MC3D_ERR_FORMAT;
        for (int32_t i = 0; i < nx; i++) {
            /* +1 so that 0 is the ambient medium; 255 + 1 -> air (:155-163) */
            int32_t t = row[i] + 1;
            if (t == 256) t = 0;
            if (t < 0 || t > 255) return MC3D_ERR_TISSUE_RANGE;
            tissue[r * nx + i] = (uint8_t)t;
        }
    }
    return MC3D_OK;
}

int mc3d_read_optprops(const char *path, int32_t *num_tissue_types, float *mua, float *mus,
                       float *g, float *n, int32_t cap)
{
    if (!path || !num_tissue_types) return MC3D_ERR_ARG;
    File f(fopen(path, "rb"));
    if (!f.f) return MC3D_ERR_IO;
    int32_t T = 0;
    if (fread(&T, sizeof T, 1, f.f) != 1) return MC3D_ERR_FORMAT;
    if (T < 1 || T > 255) return MC3D_ERR_FORMAT;
    *num_tissue_types = T + 1;
    if (!mua || !mus || !g || !n) return MC3D_OK; /* size query */
    if (T + 1 > cap) return MC3D_ERR_ARG;
    /* air at index 0 (:38-42) */
    mua[0] = 0; mus[0] = 0; g[0] = 0; n[0] = 1.0f;
    for (int32_t k = 1; k <= T; k++) {
        double rec[4];
        if (fread(rec, sizeof(double), 4, f.f) != 4) return MC3D_ERR_FORMAT;
        mua[k] = (float)rec[0];
        mus[k] = (float)rec[1];
        g[k] = (float)rec[2];
        n[k] = (float)rec[3];
    }
    return MC3D_OK;
}

int mc3d_save_property(const char *path, int32_t dims, int32_t nx, int32_t ny, int32_t nz,
                       double dx, double dy, double dz, const double *data)
{
    if (!path || !data) return MC3D_ERR_ARG;
    if (dims < 2 || dims > 3) return MC3D_ERR_ARG; /* "Unsupported number of dimensions." */
    File f(fopen(path, "wb"));
    if (!f.f) return MC3D_ERR_IO;
    /* the reference's geometry_t stores dx as float; callers pass that value */
    int ok = 1;
    ok &= fwrite(&dims, sizeof dims, 1, f.f) == 1;
    ok &= fwrite(&nx, sizeof nx, 1, f.f) == 1;
    ok &= fwrite(&ny, sizeof ny, 1, f.f) == 1;
    if (dims > 2) ok &= fwrite(&nz, sizeof nz, 1, f.f) == 1;
    ok &= fwrite(&dx, sizeof dx, 1, f.f) == 1;
    ok &= fwrite(&dy, sizeof dy, 1, f.f) == 1;
    if (dims > 2) ok &= fwrite(&dz, sizeof dz, 1, f.f) == 1;
    size_t size = (size_t)nx * ny * (dims > 2 ? nz : 1);
    ok &= fwrite(data, sizeof(double), size, f.f) == size;
    return ok ? MC3D_OK : MC3D_ERR_IO;
}

int mc3d_save_diff_refl(const char *outname, int32_t nx, int32_t ny, double dx, double dy,
                        const double *R, int64_t num_photons)
{
    if (!outname || !R || nx <= 0 || ny <= 0) return MC3D_ERR_ARG;
    std::string path = std::string(outname) + "_drs.bin";
    std::vector<double> out((size_t)nx * ny);
    for (size_t i = 0; i < out.size(); i++) out[i] = R[i] / (num_photons * 1.0);
    return mc3d_save_property(path.c_str(), 2, nx, ny, 1, dx, dy, 0.0, out.data());
}

} /* extern "C" */
