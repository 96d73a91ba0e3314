/*
 * mc3d_safedist.cu -- the safe-distance map of a voxel grid, for merged steps.
 *
 * r(v) is the largest r <= MC3D_SAFE_CAP such that every voxel of the cube of
 * half-width r (Chebyshev radius, in voxels) around v lies inside the grid and
 * has v's tissue.  A photon in voxel v can then cross that whole cube in one
 * step: the voxel-face crossings inside it change nothing in the reference's
 * step (src/mc3d_gpu.cu:181-339 with ni == nt: no Fresnel event, and no
 * absorption or scattering on a hit).
 *
 * The medium does not end at the grid's bottom face: the reference clamps the
 * voxel index (the texture's clamp addressing, src/mc3d_gpu.cu:416-418), so below
 * the grid every column continues with its last voxel.  The map therefore covers
 * nz + MC3D_SAFE_CAP slices, the extra ones standing for that continuation, and
 * only the top and lateral faces (air above, mirrors at the sides) bound it; a
 * photon deeper than the map reads its last slice, which is exact because every
 * slice below the grid is the same.
 *
 * Computation: r is the L-infinity distance transform of the boundary set B
 * (voxels on the top or lateral faces, or with one of their 26 neighbours in
 * another tissue): the nearest other-tissue voxel u of v, at Chebyshev distance
 * d, has a neighbour w of v's tissue at distance d - 1, and w is in B; so r(v) =
 * min over b in B of |v - b|_inf.  That transform is separable:
 *   D1 = distance along x to B, D2 = min_k max(|k|, D1 shifted k along y),
 *   D3 = the same along z over D2,
 * each pass scanning outward from the voxel and stopping once the offset reaches
 * the best value found, so the work per voxel is proportional to its result.
 */
#include <stdint.h>
#include "mc3d_launch.h"

namespace mc3d {

namespace {

/* B over the map's nz_map slices; tissue slice index clamped to nz - 1 */
__global__ void boundary_kernel(const uint8_t *__restrict__ t, int nx, int ny, int nz,
                                int nz_map, uint8_t *__restrict__ out)
{
    const int64_t plane = (int64_t)nx * ny;
    const int64_t nv = plane * nz_map;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % nx);
        const int j = (int)((v / nx) % ny);
        const int k = (int)(v / plane);
        bool b = i == 0 || j == 0 || k == 0 || i == nx - 1 || j == ny - 1;
        const int64_t col = (int64_t)j * nx + i;
        const uint8_t c = t[(int64_t)min(k, nz - 1) * plane + col];
        for (int dk = -1; dk <= 1 && !b; dk++) {
            const int64_t kk = (int64_t)min(k + dk, nz - 1) * plane; /* k >= 1 here */
            for (int dj = -1; dj <= 1 && !b; dj++)
                for (int di = -1; di <= 1 && !b; di++)
                    b = t[kk + col + (int64_t)dj * nx + di] != c;
        }
        out[v] = b ? 0 : MC3D_SAFE_CAP;
    }
}

/* D1(v): offset along x to the nearest voxel with in[] == 0, capped */
__global__ void pass_x_kernel(const uint8_t *__restrict__ in, int nx, int ny, int nz,
                              uint8_t *__restrict__ out)
{
    const int64_t nv = (int64_t)nx * ny * nz;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(v % nx);
        int best = MC3D_SAFE_CAP;
        for (int d = 0; d < best; d++) {
            if ((i - d >= 0 && in[v - d] == 0) || (i + d < nx && in[v + d] == 0)) {
                best = d;
                break;
            }
        }
        out[v] = (uint8_t)best;
    }
}

/* min over offsets d along an axis of max(|d|, in[v + d * stride]), capped */
__global__ void pass_minmax_kernel(const uint8_t *__restrict__ in, int nx, int ny, int nz,
                                   int axis, uint8_t *__restrict__ out)
{
    const int64_t nv = (int64_t)nx * ny * nz;
    const int64_t stride = axis == 1 ? nx : (int64_t)nx * ny;
    const int n = axis == 1 ? ny : nz;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int c = axis == 1 ? (int)((v / nx) % ny) : (int)(v / ((int64_t)nx * ny));
        int best = in[v];
        for (int d = 1; d < best; d++) {
            if (c - d >= 0) best = min(best, max(d, (int)in[v - d * stride]));
            if (c + d < n) best = min(best, max(d, (int)in[v + d * stride]));
            /* below the map (z pass only): the continuation, equal to the last slice */
            else if (axis == 2) best = min(best, max(d, (int)in[v + (int64_t)(n - 1 - c) * stride]));
        }
        out[v] = (uint8_t)best;
    }
}

/* the merged kernel's cells: tissue | box radius << 8.  r is the safe distance of
 * the tissue grid (the box holds one tissue); rn is the safe distance of the grid of
 * refractive-index classes (tissues whose index is equal in every optical set used
 * with the geometry share a class).  The box radius min(r, rn - 1) keeps a shell of
 * one voxel between the box and any index change, top face or lateral face, so
 * every reflection happens in a one-voxel step, while a box may still end at a
 * boundary between tissues of equal index, where the reference's step only moves
 * the photon on. */
__global__ void pack_kernel(const uint8_t *__restrict__ t, const uint8_t *__restrict__ r,
                            const uint8_t *__restrict__ rn, int nx, int ny, int nz, int nz_map,
                            uint16_t *__restrict__ out)
{
    const int64_t plane = (int64_t)nx * ny;
    const int64_t nv = plane * nz_map;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(v / plane);
        const int box = min((int)r[v], max((int)rn[v] - 1, 0));
        out[v] = (uint16_t)(t[(int64_t)min(k, nz - 1) * plane + v % plane] | (box << 8));
    }
}

/* each voxel's refractive-index class, from a 256-entry table */
struct ClassTable {
    uint8_t c[256];
};

__global__ void class_kernel(const uint8_t *__restrict__ t, int64_t nv,
                             const __grid_constant__ ClassTable lut, uint8_t *__restrict__ out)
{
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
         v += (int64_t)gridDim.x * blockDim.x)
        out[v] = lut.c[t[v]];
}

int grid_for(int64_t nv)
{
    int64_t want = (nv + 255) / 256;
    return (int)(want < 148 * 32 ? want : 148 * 32);
}

} /* namespace */

cudaError_t launch_safe_distance(const uint8_t *tissue, int nx, int ny, int nz, uint8_t *out,
                                 uint8_t *tmp_a, uint8_t *tmp_b, cudaStream_t stream)
{
    const int nz_map = nz + MC3D_SAFE_CAP;
    const int64_t nv = (int64_t)nx * ny * nz_map;
    if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
    const int grid = grid_for(nv);
    boundary_kernel<<<grid, 256, 0, stream>>>(tissue, nx, ny, nz, nz_map, tmp_a);
    pass_x_kernel<<<grid, 256, 0, stream>>>(tmp_a, nx, ny, nz_map, tmp_b);
    pass_minmax_kernel<<<grid, 256, 0, stream>>>(tmp_b, nx, ny, nz_map, 1, tmp_a);
    pass_minmax_kernel<<<grid, 256, 0, stream>>>(tmp_a, nx, ny, nz_map, 2, out);
    return cudaGetLastError();
}

cudaError_t launch_pack_cells(const uint8_t *tissue, const uint8_t *radius,
                              const uint8_t *radius_n, int nx, int ny, int nz, uint16_t *cells,
                              cudaStream_t stream)
{
    const int nz_map = nz + MC3D_SAFE_CAP;
    const int64_t nv = (int64_t)nx * ny * nz_map;
    if (nx <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
    pack_kernel<<<grid_for(nv), 256, 0, stream>>>(tissue, radius, radius_n, nx, ny, nz, nz_map,
                                                  cells);
    return cudaGetLastError();
}

cudaError_t launch_index_classes(const uint8_t *tissue, int64_t nv, const uint8_t *classes,
                                 uint8_t *out, cudaStream_t stream)
{
    if (nv <= 0) return cudaSuccess;
    ClassTable lut;
    for (int t = 0; t < 256; t++) lut.c[t] = classes[t];
    class_kernel<<<grid_for(nv), 256, 0, stream>>>(tissue, nv, lut, out);
    return cudaGetLastError();
}

} /* namespace mc3d */
