"""Statistics for comparing two simulations of the same physics.

A reflectance bin's estimate is R = sum W / N with variance (sum W^2 / N - R^2) / N
(the per-photon weights of a bin are independent), which is why every run keeps
sum W^2 per bin (drs_sq).  Two runs of the same physics with independent seeds
then differ bin by bin by z = (R_a - R_b) / sqrt(var_a + var_b), a standard
normal, and sum z^2 over bins follows a chi-square law.
"""
from __future__ import annotations

import numpy as np

from . import WEIGHT_SCALE


def superbin(a: np.ndarray, f: int) -> np.ndarray:
    """sum f x f blocks of a [ny, nx] array (ragged edges dropped)"""
    ny, nx = a.shape
    return a[: ny - ny % f, : nx - nx % f].reshape(ny // f, f, nx // f, f).sum(axis=(1, 3))


def drs_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b, f=8, min_mean=1e-5) -> np.ndarray:
    """Per-(super)bin z-scores of reflectance between two runs, for bins whose mean
    reflectance exceeds min_mean and whose variance is positive."""
    sa = superbin(np.asarray(sum_a, np.float64), f) / WEIGHT_SCALE
    qa = superbin(np.asarray(sq_a, np.float64), f) / WEIGHT_SCALE
    sb = superbin(np.asarray(sum_b, np.float64), f) / WEIGHT_SCALE
    qb = superbin(np.asarray(sq_b, np.float64), f) / WEIGHT_SCALE
    ra, rb = sa / n_a, sb / n_b
    va = np.maximum(qa / n_a - ra ** 2, 0) / n_a
    vb = np.maximum(qb / n_b - rb ** 2, 0) / n_b
    ok = ((ra + rb) / 2 > min_mean) & (va + vb > 0)
    return (ra[ok] - rb[ok]) / np.sqrt(va[ok] + vb[ok])


def drs_chi2(sum_a, sq_a, n_a, sum_b, sq_b, n_b, f=8, min_mean=1e-5):
    """(chi2, dof, p) of the per-(super)bin z-scores (drs_z)."""
    from scipy import stats
    z = drs_z(sum_a, sq_a, n_a, sum_b, sq_b, n_b, f, min_mean)
    chi2, dof = float(np.sum(z * z)), int(z.size)
    return chi2, dof, float(stats.chi2.sf(chi2, dof)) if dof else 1.0


def total_z(ta: dict, tb: dict, key="r_in") -> float:
    """z-score of a total weight fraction between two runs (binomial-like variance,
    an upper bound since every photon's weight is at most 1)."""
    fa = ta[key] / WEIGHT_SCALE / ta["photons"]
    fb = tb[key] / WEIGHT_SCALE / tb["photons"]
    va = fa * (1 - min(fa, 1)) / ta["photons"] + 1e-30
    vb = fb * (1 - min(fb, 1)) / tb["photons"] + 1e-30
    return float((fa - fb) / np.sqrt(va + vb))
