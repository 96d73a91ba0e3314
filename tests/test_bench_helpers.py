"""The sweep measurement's helpers in bench.py, on CPU: the reference arm's
stratified subset of the 128 wavelengths, the strata it estimates the whole
sweep from, and the total-reflectance sigma taken from the bins' sum W^2."""
from __future__ import annotations

import numpy as np

import bench
import ymc3d_b200 as m
from ymc3d_b200 import workloads as W


def test_subset_is_one_seeded_job_per_mua_stratum():
    w = W.sweep(photon_scale=1.0, beam="uniform")
    strata = bench.sweep_strata(w)
    assert len(strata) == bench.SWEEP_STRATA
    flat = sorted(k for s in strata for k in s)
    assert flat == list(range(len(w.jobs)))  # a partition of the jobs
    mua = [float(w.props[j.props].mua[1]) for j in w.jobs]
    for a, b in zip(strata, strata[1:]):
        assert max(mua[k] for k in a) <= min(mua[k] for k in b)  # ordered by mua
    sub = bench.sweep_subset(w)
    assert sub == bench.sweep_subset(w)  # seeded
    assert [next(i for i, s in enumerate(strata) if k in s) for k in sub] == list(
        range(bench.SWEEP_STRATA))


def test_total_reflectance_sigma_from_bins():
    """each photon's reflected weight lands in one bin, so the bins' sums give the
    photons' mean and standard error of the total"""
    rng = np.random.default_rng(3)
    n = 20000
    w = rng.uniform(0, 1, n) * (rng.uniform(size=n) < 0.6)  # 60 % reflected
    bins = rng.integers(0, 16, n)
    q = np.round(w * m.WEIGHT_SCALE).astype(np.uint64)
    q2 = np.round(w * w * m.WEIGHT_SCALE).astype(np.uint64)
    drs = np.bincount(bins, weights=q, minlength=16).astype(np.uint64).reshape(4, 4)
    sq = np.bincount(bins, weights=q2, minlength=16).astype(np.uint64).reshape(4, 4)
    r = m.Result(drs, sq, np.zeros_like(drs), {"photons": n})
    mean, sigma = bench.r_total_sigma(r)
    assert abs(mean - w.mean()) < 1e-6
    assert abs(sigma - w.std() / np.sqrt(n)) / sigma < 1e-3
