// The file a maintainer adds to the reference's build in place of src/mc3d_gpu.cu:
// run_3dmc_gpu (src/mc3d_gpu.h:16) forwarded to libmc3d.so's mc3d_run_3dmc_gpu.
// Compiled by nvcc like the reference's other sources (src/mc3d_types.h pulls in
// gpumcml_rng.h, which uses __device__).  src/mc3d_photons.cu leaves the build with
// src/mc3d_gpu.cu: its photon_detector needs photontrack_get_grid_coord from there,
// and the library does that work on the device.  oracle/build_ref.py links this file
// with the reference's src/mc3d_main.cu and src/mc3d_io.cu into _ref/gpu-mc-bridge,
// the reference's own command line running on the library.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "mc3d_types.h"
#include "mc3d.h"          // from ymc3d-b200/include

void run_3dmc_gpu(geometry_t geometry, opticalprops_t optProps, int num_photons,
                  double *R, double *R_tot, double *T, double *T_tot, float *A,
                  int *num_finished_photons)
{
    mc3d_ref_geometry g;
    mc3d_ref_opticalprops p;
    static_assert(sizeof g == sizeof geometry, "geometry_t layout");
    memcpy(&g, &geometry, sizeof g);
    p.num_tissue_types = optProps.num_tissue_types;
    p.n = optProps.n; p.mua = optProps.mua; p.mus = optProps.mus; p.g = optProps.g;
    p.alloc_where = (int)optProps.allocWhere;
    int st = mc3d_run_3dmc_gpu(g, p, num_photons, R, R_tot, T, T_tot, A,
                               num_finished_photons);
    if (st != MC3D_OK) {                       // the reference exits on a missing table
        fprintf(stderr, "%s\n", mc3d_last_error());
        exit(1);
    }
}
