/*
 * io_harness.cu -- C entry points into the reference's own file I/O
 * (src/mc3d_io.cu, compiled unmodified where it lies).
 *
 * TEST INFRASTRUCTURE ONLY: golden readers/writers for the format tests.
 */
#include <cstring>
#include "mc3d_types.h"
#include "mc3d_io.h"

/* geometry_read_from_file; copies the remapped tissue array when `tissue` is set */
extern "C" int ref_read_geometry(const char *path, int *n3, float *d3, int *tissue,
                                 long long cap)
{
    geometry_t g;
    memset(&g, 0, sizeof g);
    if (geometry_read_from_file(&g, (char *)path) != 0) return -1;
    n3[0] = g.num_x; n3[1] = g.num_y; n3[2] = g.num_z;
    d3[0] = g.sample_dx; d3[1] = g.sample_dy; d3[2] = g.sample_dz;
    long long nv = (long long)g.num_x * g.num_y * g.num_z;
    if (tissue && nv <= cap) memcpy(tissue, g.tissue_type, sizeof(int) * nv);
    geometry_free(&g);
    return 0;
}

extern "C" int ref_read_optprops(const char *path, int *ntypes, float *mua, float *mus, float *g,
                                 float *n, int cap)
{
    opticalprops_t p;
    memset(&p, 0, sizeof p);
    if (opticalprops_read_from_file(&p, (char *)path) != 0) return -1;
    *ntypes = p.num_tissue_types;
    if (mua && p.num_tissue_types <= cap) {
        memcpy(mua, p.mua, sizeof(float) * p.num_tissue_types);
        memcpy(mus, p.mus, sizeof(float) * p.num_tissue_types);
        memcpy(g, p.g, sizeof(float) * p.num_tissue_types);
        memcpy(n, p.n, sizeof(float) * p.num_tissue_types);
    }
    opticalprops_free(&p);
    return 0;
}

/* save_diff_refl for a geometry of the given size and (float) voxel size */
extern "C" void ref_save_diff_refl(int nx, int ny, float dx, float dy, const double *R,
                                   int num_photons, const char *outname)
{
    geometry_t g;
    memset(&g, 0, sizeof g);
    g.num_x = nx; g.num_y = ny; g.num_z = 1;
    g.sample_dx = dx; g.sample_dy = dy; g.sample_dz = 1;
    save_diff_refl(g, (double *)R, num_photons, (char *)outname);
}
