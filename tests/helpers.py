"""Helpers shared by the parity tests."""
from __future__ import annotations

import numpy as np

import oracle
import ymc3d_b200 as m


def oracle_job(geom: m.Geometry, props: m.OpticalProps, job: m.Job, table, threads=0,
               photon_log=False, first=0, count=-1, max_steps=0, absorption_map=False):
    return oracle.run(geom.tissue, geom.dx, geom.dy, geom.dz, props.mua, props.mus, props.g,
                      props.n, int(job.photons), job.num_streams(), int(job.seed), table,
                      beam=m.BEAMS[job.beam], threads=threads, first=first, count=count,
                      max_steps=max_steps, photon_log=photon_log,
                      absorption_map=absorption_map)


def residual(t: dict) -> int:
    return int(t["w_launched"]) - (int(t["r_in"]) + int(t["r_out"]) + int(t["t_in"]) +
                                   int(t["t_out"]) + int(t["absorbed"]) + int(t["rr_killed"]) -
                                   int(t["rr_created"]) + int(t["lost"]))


# the comparison statistics live in the package (bench.py uses them too)
from ymc3d_b200.stats import drs_chi2, superbin, total_z  # noqa: E402,F401


def safe_distance_bruteforce(t: np.ndarray, cap: int = 63) -> np.ndarray:
    """Definition of the merged-step safe-distance map, checked cube by cube: on
    the grid extended below by copies of its last slice (the clamped
    continuation), per voxel the largest r <= cap such that the Chebyshev cube of
    half-width r is uniform, below the top face and inside the lateral faces."""
    from scipy.ndimage import maximum_filter, minimum_filter
    nz, ny, nx = t.shape
    ext = np.concatenate([t, np.repeat(t[-1:], cap, axis=0)]).astype(np.int16)
    k, j, i = np.meshgrid(np.arange(nz + cap), np.arange(ny), np.arange(nx), indexing="ij")
    out = np.zeros(ext.shape, np.uint8)
    alive = np.ones(ext.shape, bool)
    for q in range(1, cap + 1):
        size = 2 * q + 1
        inside = (k - q >= 0) & (j - q >= 0) & (i - q >= 0) & (j + q < ny) & (i + q < nx)
        uniform = (maximum_filter(ext, size, mode="nearest") ==
                   minimum_filter(ext, size, mode="nearest"))
        alive &= inside & uniform
        if not alive.any():
            break
        out[alive] = q
    return out
