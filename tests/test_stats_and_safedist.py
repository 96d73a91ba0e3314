"""CPU checks of the pieces the GPU tests lean on: the cube-by-cube definition of
the merged-step safe-distance map (hand-worked cases) and the comparison
statistics of ymc3d_b200.stats (their null distribution on synthetic runs)."""
from __future__ import annotations

import numpy as np

from helpers import safe_distance_bruteforce
from ymc3d_b200 import WEIGHT_SCALE, stats


def test_safe_distance_definition_by_hand():
    t = np.ones((9, 9, 9), np.uint8)
    r = safe_distance_bruteforce(t)
    assert r.shape == (9 + 63, 9, 9)
    # lateral faces and the top bound the cube; the bottom is open
    assert r[4, 4, 4] == 4 and r[0, 4, 4] == 0 and r[1, 4, 4] == 1 and r[4, 4, 0] == 0
    assert r[8, 4, 4] == 4 and r[70, 4, 4] == 4
    t[4, 4, 4] = 2
    r = safe_distance_bruteforce(t)
    assert r[4, 4, 4] == 0          # its 26 neighbours differ
    assert r[2, 2, 2] == 1          # Chebyshev distance 2 to the odd voxel
    assert r[4, 4, 7] == 1          # limited by the lateral face, not the odd voxel


def test_safe_distance_layers():
    t = np.ones((20, 30, 30), np.uint8)
    t[10:] = 2                      # an interface between slices 9 and 10
    r = safe_distance_bruteforce(t)
    assert r[9, 15, 15] == 0 and r[10, 15, 15] == 0
    assert r[5, 15, 15] == 4        # 5 to the top face, 4 to the last slice of its layer
    assert r[19 + 20, 15, 15] == 14  # the continuation below: only the sides bound it


def _fake_run(rng, n, p_bins, w_mean=0.3):
    """tallies of n photons, each landing in a bin with probability p_bins with a
    random weight; returns (sum Q(W), sum Q(W^2), totals)"""
    bins = p_bins.size
    which = rng.choice(bins + 1, size=n, p=np.append(p_bins, 1 - p_bins.sum()))
    w = rng.uniform(0, 2 * w_mean, size=n)
    hit = which < bins
    s = np.bincount(which[hit], weights=w[hit], minlength=bins)
    q = np.bincount(which[hit], weights=w[hit] ** 2, minlength=bins)
    drs = np.round(s * WEIGHT_SCALE).astype(np.uint64).reshape(16, 16)
    sq = np.round(q * WEIGHT_SCALE).astype(np.uint64).reshape(16, 16)
    tot = {"photons": n, "r_in": int(drs.sum()), "absorbed": int(np.round((w[~hit]).sum() *
                                                                          WEIGHT_SCALE))}
    return drs, sq, tot


def test_chi2_null_distribution():
    rng = np.random.default_rng(12)
    p_bins = rng.dirichlet(np.ones(256)) * 0.6
    ps, zs = [], []
    for _ in range(40):
        a = _fake_run(rng, 20000, p_bins)
        b = _fake_run(rng, 30000, p_bins)
        chi2, dof, p = stats.drs_chi2(a[0], a[1], 20000, b[0], b[1], 30000, f=2)
        assert dof == 64
        ps.append(p)
        zs.append(stats.total_z(a[2], b[2], "r_in"))
    # same physics: p-values roughly uniform; the total's z-score uses an upper
    # bound of the variance (weights <= 1), so its spread is at most about one
    assert 0.2 < np.mean(ps) < 0.8 and min(ps) > 1e-4
    assert np.std(zs) < 1.3


def test_chi2_detects_a_shift():
    rng = np.random.default_rng(13)
    p_bins = rng.dirichlet(np.ones(256)) * 0.6
    q_bins = p_bins.copy()
    q_bins[:128] *= 1.1
    a = _fake_run(rng, 200000, p_bins)
    b = _fake_run(rng, 200000, q_bins)
    chi2, dof, p = stats.drs_chi2(a[0], a[1], 200000, b[0], b[1], 200000, f=2)
    assert p < 1e-6
