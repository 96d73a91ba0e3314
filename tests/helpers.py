"""Helpers shared by the parity tests."""
from __future__ import annotations

import numpy as np
from scipy import stats

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


def superbin(a: np.ndarray, f: int) -> np.ndarray:
    ny, nx = a.shape
    return a[: ny - ny % f, : nx - nx % f].reshape(ny // f, f, nx // f, f).sum(axis=(1, 3))


def drs_chi2(sum_a, sq_a, n_a, sum_b, sq_b, n_b, f=8, min_mean=1e-5):
    """Chi-square of per-(super)bin reflectance R = sum W / N between two runs,
    each bin's variance from its own sum W^2: returns (chi2, dof, p)."""
    sa = superbin(sum_a.astype(np.float64), f) / m.WEIGHT_SCALE
    qa = superbin(sq_a.astype(np.float64), f) / m.WEIGHT_SCALE
    sb = superbin(sum_b.astype(np.float64), f) / m.WEIGHT_SCALE
    qb = superbin(sq_b.astype(np.float64), f) / m.WEIGHT_SCALE
    ra, rb = sa / n_a, sb / n_b
    va = np.maximum(qa / n_a - ra ** 2, 0) / n_a
    vb = np.maximum(qb / n_b - rb ** 2, 0) / n_b
    ok = ((ra + rb) / 2 > min_mean) & (va + vb > 0)
    chi2 = float(np.sum((ra[ok] - rb[ok]) ** 2 / (va[ok] + vb[ok])))
    dof = int(ok.sum())
    return chi2, dof, float(stats.chi2.sf(chi2, dof)) if dof else 1.0


def total_z(ta: dict, tb: dict, key="r_in"):
    """z-score of a total weight fraction between two runs (binomial-like variance
    bounded by the per-photon weight <= 1)."""
    fa = ta[key] / m.WEIGHT_SCALE / ta["photons"]
    fb = tb[key] / m.WEIGHT_SCALE / tb["photons"]
    va = fa * (1 - min(fa, 1)) / ta["photons"] + 1e-30
    vb = fb * (1 - min(fb, 1)) / tb["photons"] + 1e-30
    return (fa - fb) / np.sqrt(va + vb)


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
