"""Merged steps (MC3D_STEPS_MERGED, the fast-math default): the safe-distance map
against its brute-force definition, and merged against per-face stepping on the
same physics -- statistically equal tallies, exact conservation, fewer steps."""
from __future__ import annotations

import numpy as np
import pytest

import ymc3d_b200 as m
from helpers import drs_chi2, residual, safe_distance_bruteforce, total_z

pytestmark = pytest.mark.gpu


def _grids():
    rng = np.random.default_rng(5)
    yield np.ones((1, 1, 1), np.uint8)
    yield np.ones((3, 1, 7), np.uint8)
    yield np.ones((20, 18, 22), np.uint8)
    blocky = np.kron(rng.integers(1, 4, (3, 4, 3)), np.ones((6, 5, 7), np.int64)).astype(np.uint8)
    yield blocky
    speckled = np.ones((16, 24, 20), np.uint8)
    speckled[rng.random(speckled.shape) < 0.01] = 2
    yield speckled
    from ymc3d_b200.workloads import layered_vessel_geometry
    yield layered_vessel_geometry(40, 36, 30, 0.08).tissue


@pytest.mark.parametrize("k", range(6))
def test_safe_distance_matches_definition(engine, k):
    t = list(_grids())[k]
    assert np.array_equal(m.safe_distance(t), safe_distance_bruteforce(t))


def test_safe_distance_cap(engine):
    t = np.ones((140, 140, 140), np.uint8)
    r = m.safe_distance(t)
    assert r.shape == (140 + 63, 140, 140)
    assert r.max() == 63 and r[70, 70, 70] == 63 and r[200, 70, 70] == 63
    assert r[0].max() == 0 and r[5, 70, 70] == 5 and r[70, 70, 133] == 6
    assert r[139, 70, 70] == 63  # the bottom face is open: the medium continues


def layered_small():
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    return layered_vessel_geometry(64, 64, 32, 0.08), m.OpticalProps.from_tissues(LAYER_ROWS)


@pytest.mark.parametrize("beam", ["uniform", "pencil"])
def test_merged_vs_voxel_steps_chi2(table, beam):
    g, p = layered_small()
    mer = m.run([g], [p], [m.Job(0, 0, 2_000_000, 31, beam)], table=table)[0]
    vox = m.run([g], [p], [m.Job(0, 0, 2_000_000, 32, beam)], table=table, steps="voxel")[0]
    chi2, dof, pv = drs_chi2(mer.drs, mer.drs_sq, mer.photons, vox.drs, vox.drs_sq, vox.photons,
                             f=4 if beam == "pencil" else 8)
    assert dof > 20 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "t_in", "absorbed"):
        assert abs(total_z(mer.totals, vox.totals, key)) < 5, key
    assert mer.totals["steps"] < vox.totals["steps"]


def test_merged_steps_homogeneous_slab(table):
    """a thick uniform slab, where nearly every flight is merged"""
    g = m.Geometry(np.ones((60, 80, 80), np.uint8), 0.05, 0.05, 0.05)
    p = m.OpticalProps.from_tissues([(0.02, 8.0, 0.9, 1.37)])
    mer = m.run([g], [p], [m.Job(0, 0, 2_000_000, 41, "pencil")], table=table)[0]
    vox = m.run([g], [p], [m.Job(0, 0, 2_000_000, 42, "pencil")], table=table,
                steps="voxel")[0]
    chi2, dof, pv = drs_chi2(mer.drs, mer.drs_sq, mer.photons, vox.drs, vox.drs_sq, vox.photons,
                             f=2)
    assert dof > 100 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "t_in", "absorbed"):
        assert abs(total_z(mer.totals, vox.totals, key)) < 5, key
    assert mer.totals["steps"] * 2 < vox.totals["steps"]


def test_merged_steps_conservation_and_absorption_map(table):
    g, p = layered_small()
    r = m.run([g], [p], [m.Job(0, 0, 500_000, 77, "uniform")], table=table,
              absorption_map=True)[0]
    t = r.totals
    assert t["photons"] == 500_000 and residual(t) == 0
    assert int(r.drs.sum()) == t["r_in"] and int(r.trans.sum()) == t["t_in"]
    assert int(r.absorption.sum()) == t["absorbed"]


def test_exact_math_ignores_step_mode(table):
    g, p = layered_small()
    job = m.Job(0, 0, 20_000, 9, "uniform")
    a = m.run([g], [p], [job], table=table, math="exact")[0]
    b = m.run([g], [p], [job], table=table, math="exact", steps="voxel")[0]
    assert a.totals == b.totals and np.array_equal(a.drs, b.drs)


def test_merged_steps_absorption_profile(table):
    """the absorption map books each interaction in the voxel where it happens:
    its depth profile agrees with per-face stepping"""
    g, p = layered_small()
    mer = m.run([g], [p], [m.Job(0, 0, 1_000_000, 51, "uniform")], table=table,
                absorption_map=True)[0]
    vox = m.run([g], [p], [m.Job(0, 0, 1_000_000, 52, "uniform")], table=table,
                absorption_map=True, steps="voxel")[0]
    a = mer.absorption.sum(axis=(1, 2)).astype(np.float64) / mer.totals["w_launched"]
    b = vox.absorption.sum(axis=(1, 2)).astype(np.float64) / vox.totals["w_launched"]
    big = b > 0.01 * b.max()
    assert big.sum() > 5
    assert np.max(np.abs(a[big] - b[big]) / b[big]) < 0.05


def deep_like(nx=512, ny=512, nz=64, d=0.01):
    """a long-path, high-albedo medium like the deep-grid workload, one tissue"""
    g = m.Geometry(np.ones((nz, ny, nx), np.uint8), d, d, d)
    return g, m.OpticalProps.from_tissues([(0.001, 20.0, 0.9, 1.4)])


def test_merged_quickfix_loss_matches_voxel_steps(table):
    """The reference's end-of-chunk quickfix (src/mc3d_gpu.cu:343-353) kills a photon
    whose 45th step had db == 0: in float a scattering move can round onto a voxel
    face, and when the new direction points back across it the next one-voxel DDA
    gives 0.  On long-path media that costs a few 1e-3 of the launched weight.
    Merged steps evaluate the same one-voxel condition at the chunk's last step, so
    they lose as many photons and as much weight as per-face steps (within Poisson
    error), although the merged box itself rarely has a zero boundary distance."""
    g, p = deep_like()
    n = 1_000_000
    mer = m.run([g], [p], [m.Job(0, 0, n, 61, "uniform")], table=table)[0]
    vox = m.run([g], [p], [m.Job(0, 0, n, 62, "uniform")], table=table, steps="voxel")[0]
    qm, qv = mer.totals["quickfix"], vox.totals["quickfix"]
    assert qv > 1000, qv
    assert abs(qm - qv) < 4 * np.sqrt(qm + qv), (qm, qv)
    lm = mer.totals["lost"] / m.WEIGHT_SCALE / n
    lv = vox.totals["lost"] / m.WEIGHT_SCALE / n
    assert lv > 1e-4
    # each lost weight is at most 1: the Poisson count bounds the variance
    assert abs(lm - lv) < 4 * np.sqrt(qm + qv) / n, (lm, lv)
    for key in ("r_in", "r_out", "absorbed"):
        assert abs(total_z(mer.totals, vox.totals, key)) < 5, key
    assert residual(mer.totals) == 0 and residual(vox.totals) == 0


def test_merged_vs_voxel_many_interfaces(table):
    """Blocks of four tissues with different refractive indices and in-volume air:
    most reflections (Fresnel, lateral mirror, total internal reflection at the
    air) happen next to a tissue boundary, where merged steps shrink to one-voxel
    steps.  Both step modes must give the same DRS, totals and quickfix losses."""
    rng = np.random.default_rng(11)
    coarse = rng.integers(1, 5, (6, 8, 8)).astype(np.uint8)
    t = np.kron(coarse, np.ones((6, 6, 6), np.uint8))
    t[rng.random(t.shape) < 0.002] = 0  # scattered in-volume air voxels
    t[:3] = 1  # a uniform top layer
    g = m.Geometry(t, 0.02, 0.02, 0.02)
    p = m.OpticalProps.from_tissues([(0.05, 15.0, 0.85, 1.37), (0.2, 20.0, 0.9, 1.44),
                                     (0.02, 10.0, 0.8, 1.50), (1.0, 25.0, 0.95, 1.33)])
    n = 2_000_000
    mer = m.run([g], [p], [m.Job(0, 0, n, 71, "uniform")], table=table)[0]
    vox = m.run([g], [p], [m.Job(0, 0, n, 72, "uniform")], table=table, steps="voxel")[0]
    chi2, dof, pv = drs_chi2(mer.drs, mer.drs_sq, mer.photons, vox.drs, vox.drs_sq, vox.photons,
                             f=4)
    assert dof > 100 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "t_in", "absorbed"):
        assert abs(total_z(mer.totals, vox.totals, key)) < 5, key
    assert mer.totals["fresnel"] > 0 and mer.totals["t_in"] > 0
    qm, qv = mer.totals["quickfix"], vox.totals["quickfix"]
    assert abs(qm - qv) < 4 * np.sqrt(qm + qv + 1), (qm, qv)
    # Fresnel events per photon agree too: every one is a one-voxel step
    fm, fv = mer.totals["fresnel"], vox.totals["fresnel"]
    assert abs(fm - fv) < 0.02 * fv, (fm, fv)
    assert residual(mer.totals) == 0 and mer.totals["steps"] < vox.totals["steps"]


def test_merged_boxes_cross_equal_index_boundaries(table):
    """Blobs of three tissues with one refractive index and a fourth with another
    (and in-volume air): merged boxes may end at the equal-index boundaries, where
    the reference's step only moves the photon into the next tissue's
    coefficients, but keep their one-voxel margin at the index change.  Merged and
    per-face steps agree in DRS, totals, Fresnel events and quickfix losses, and
    the equal-index boundaries cost fewer merged steps than distinct indices do."""
    rng = np.random.default_rng(12)
    t = np.kron(rng.integers(1, 5, (5, 6, 6)), np.ones((8, 8, 8), np.int64)).astype(np.uint8)
    t[rng.random(t.shape) < 0.001] = 0
    g = m.Geometry(t, 0.01, 0.01, 0.01)
    same = [(0.001, 20.0, 0.9, 1.4), (0.0012, 18.0, 0.9, 1.4), (0.0009, 22.0, 0.9, 1.4),
            (0.002, 20.0, 0.9, 1.33)]
    p = m.OpticalProps.from_tissues(same)
    n = 1_000_000
    mer = m.run([g], [p], [m.Job(0, 0, n, 81, "uniform")], table=table)[0]
    vox = m.run([g], [p], [m.Job(0, 0, n, 82, "uniform")], table=table, steps="voxel")[0]
    chi2, dof, pv = drs_chi2(mer.drs, mer.drs_sq, mer.photons, vox.drs, vox.drs_sq, vox.photons,
                             f=4)
    assert dof > 100 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "t_in", "absorbed"):
        assert abs(total_z(mer.totals, vox.totals, key)) < 5, key
    qm, qv = mer.totals["quickfix"], vox.totals["quickfix"]
    assert abs(qm - qv) < 4 * np.sqrt(qm + qv + 1), (qm, qv)
    fm, fv = mer.totals["fresnel"], vox.totals["fresnel"]
    assert abs(fm - fv) < 4 * np.sqrt(fm + fv), (fm, fv)
    assert residual(mer.totals) == 0
    # with four distinct indices the same grid merges fewer of its per-face steps
    distinct = m.OpticalProps.from_tissues([(a, b, c, 1.30 + 0.05 * k)
                                            for k, (a, b, c, _) in enumerate(same)])
    dj = m.Job(0, 0, 200_000, 83, "uniform")
    dm = m.run([g], [distinct], [dj], table=table)[0]
    dv = m.run([g], [distinct], [dj], table=table, steps="voxel")[0]
    same_ratio = mer.totals["steps"] / vox.totals["steps"]
    distinct_ratio = dm.totals["steps"] / dv.totals["steps"]
    assert same_ratio < 0.95 * distinct_ratio, (same_ratio, distinct_ratio)
