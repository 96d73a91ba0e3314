"""Precision study: FP32 transport (the reference's precision) against the same
photon loop in FP64, stated as a chi-square over DRS bins and as z-scores of the
totals.  CPU part: the FP32 oracle against its FP64 build.  GPU part: the FP64
engine (MC3D_MATH_F64) against the FP64 oracle, which pins it, and the fast FP32
engine against both, on a long-path, high-albedo medium like the 1024x1024x256
precision workload (mua 0.001/mm, mus 20/mm, g 0.9, n 1.4)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle
import ymc3d_b200 as m
from helpers import drs_chi2, residual, total_z


def deep_like(n=48, d=0.01, mua=0.01):
    g = m.Geometry(np.ones((n, n, n), np.uint8), d, d, d)
    p = m.OpticalProps.from_tissues([(mua, 20.0, 0.9, 1.4)])
    return g, p


def run_oracle(g, p, photons, seed, table, f64, beam=1):
    return oracle.run(g.tissue, g.dx, g.dy, g.dz, p.mua, p.mus, p.g, p.n, photons, photons,
                      seed, table, beam=beam, threads=0, f64=f64)


def test_fp32_vs_fp64_oracle(orc, table):
    g, p = deep_like(32, 0.02, 0.05)
    a = run_oracle(g, p, 20000, 101, table, False)
    b = run_oracle(g, p, 20000, 202, table, True)
    chi2, dof, pv = drs_chi2(a["drs"], a["drs_sq"], 20000, b["drs"], b["drs_sq"], 20000, f=4)
    assert dof > 10 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "absorbed"):
        assert abs(total_z(a["totals"], b["totals"], key)) < 5


@pytest.mark.gpu
def test_fast_fp32_engine_vs_fp64_oracle(table):
    g, p = deep_like(48, 0.01, 0.01)
    o = run_oracle(g, p, 30000, 303, table, True)
    r = m.run([g], [p], [m.Job(0, 0, 2_000_000, 404, "pencil")], table=table)[0]
    chi2, dof, pv = drs_chi2(r.drs, r.drs_sq, r.photons, o["drs"], o["drs_sq"],
                             o["totals"]["photons"], f=4)
    assert dof > 10 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "absorbed"):
        assert abs(total_z(r.totals, o["totals"], key)) < 5, key


@pytest.mark.gpu
@pytest.mark.parametrize("steps", ["voxel", "merged"])
def test_f64_engine_vs_fp64_oracle(table, steps):
    """the FP64 engine follows the FP64 transcription (statistically: CUDA's and
    libm's double functions differ in the last bit, and trajectories part)"""
    g, p = deep_like(48, 0.01, 0.01)
    o = run_oracle(g, p, 30000, 505, table, True)
    r = m.run([g], [p], [m.Job(0, 0, 1_000_000, 606, "pencil")], table=table, math="f64",
              steps=steps)[0]
    assert residual(r.totals) == 0 and r.photons == 1_000_000
    chi2, dof, pv = drs_chi2(r.drs, r.drs_sq, r.photons, o["drs"], o["drs_sq"],
                             o["totals"]["photons"], f=4)
    assert dof > 10 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "absorbed"):
        assert abs(total_z(r.totals, o["totals"], key)) < 5, key


@pytest.mark.gpu
@pytest.mark.parametrize("steps", ["merged", "voxel"])
def test_fast_fp32_engine_vs_f64_engine(table, steps):
    """FP32 against FP64 stepping at 2e6 photons a side: the per-bin differences
    stay within sampling error (chi-square) and the totals within 5 sigma"""
    g, p = deep_like(48, 0.01, 0.01)
    a = m.run([g], [p], [m.Job(0, 0, 2_000_000, 707, "pencil")], table=table, steps=steps)[0]
    b = m.run([g], [p], [m.Job(0, 0, 2_000_000, 808, "pencil")], table=table, math="f64",
              steps=steps)[0]
    chi2, dof, pv = drs_chi2(a.drs, a.drs_sq, a.photons, b.drs, b.drs_sq, b.photons, f=2)
    assert dof > 100 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "t_in", "absorbed"):
        assert abs(total_z(a.totals, b.totals, key)) < 5, key
