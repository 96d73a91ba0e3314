"""Bit-exact parity: the engine's exact-math kernel against the CPU oracle.

With correctly rounded arithmetic and the shared series functions, every photon
of the engine must end in exactly the state the oracle's restatement of
src/mc3d_gpu.cu:74-376 computes, and every tally must be identical."""
from __future__ import annotations

import numpy as np
import pytest

import ymc3d_b200 as m
from helpers import oracle_job, residual

pytestmark = pytest.mark.gpu


def _compare(geoms, props, jobs, table, **kw):
    res = m.run(geoms, props, jobs, table=table, math="exact", photon_log=True, **kw)
    for r, job in zip(res, jobs):
        o = oracle_job(geoms[job.geom], props[job.props], job, table, photon_log=True,
                       max_steps=kw.get("max_steps", 0))
        assert len(r.photon_log) == len(o["photon_log"]) == job.photons
        a = r.photon_log.view(np.uint8).reshape(len(r.photon_log), 48)
        b = o["photon_log"].view(np.uint8).reshape(len(o["photon_log"]), 48)
        bad = np.nonzero((a != b).any(axis=1))[0]
        assert bad.size == 0, (f"{bad.size} photons differ, first {bad[:5]}:\n"
                               f"engine {r.photon_log[bad[:3]]}\noracle {o['photon_log'][bad[:3]]}")
        assert r.totals == o["totals"]
        assert np.array_equal(r.drs, o["drs"])
        assert np.array_equal(r.drs_sq, o["drs_sq"])
        assert np.array_equal(r.trans, o["trans"])
        assert residual(r.totals) == 0
    return res


def homogeneous(n=32, d=0.1, row=(0.01, 10.0, 0.9, 1.4)):
    return m.Geometry(np.ones((n, n, n), np.uint8), d, d, d), m.OpticalProps.from_tissues([row])


def layered(nx=64, ny=64, nz=32, d=0.08, air_holes=False):
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    g = layered_vessel_geometry(nx, ny, nz, d)
    if air_holes:
        g.tissue[nz // 2: nz // 2 + 3, 10:20, 10:20] = 0  # in-volume air (file value 255)
    return g, m.OpticalProps.from_tissues(LAYER_ROWS)


@pytest.mark.parametrize("beam,streams", [("pencil", 0), ("pencil", 97), ("uniform", 0),
                                          ("uniform", 250)])
def test_homogeneous(table, beam, streams):
    g, p = homogeneous()
    _compare([g], [p], [m.Job(0, 0, 2000, 1796308352, beam, streams)], table)


def test_layered_vessel_fresnel(table):
    g, p = layered()
    r = _compare([g], [p], [m.Job(0, 0, 3000, 424242, "uniform")], table)
    assert r[0].totals["fresnel"] > 0


def test_in_volume_air_transmission(table):
    g, p = layered(air_holes=True)
    r = _compare([g], [p], [m.Job(0, 0, 3000, 31337, "uniform")], table)
    assert r[0].totals["t_in"] + r[0].totals["t_out"] > 0


def test_g_zero_quickfix_path(table):
    """g = 0 makes the reference's Henyey-Greenstein step 0 * inf = NaN; the
    photon goes non-finite and the end-of-launch quickfix zeroes it"""
    g, p = homogeneous(16, 0.1, (0.1, 5.0, 0.0, 1.4))
    r = _compare([g], [p], [m.Job(0, 0, 500, 777, "uniform")], table)
    assert r[0].totals["quickfix"] > 0


def test_step_cap(table):
    g, p = homogeneous()
    r = _compare([g], [p], [m.Job(0, 0, 1000, 99, "pencil")], table, max_steps=60)
    assert r[0].totals["capped"] > 0


def test_rejection_heavy_table():
    small = np.array([4294967118] + [3, 5, 7, 11, 13, 17] * 50, np.uint32)
    g, p = homogeneous(16)
    _compare([g], [p], [m.Job(0, 0, 1500, 55555, "uniform")], small)


def test_batched_jobs(table):
    g1, p1 = homogeneous(24, 0.1)
    g2, p2 = layered(48, 40, 24, 0.1)
    jobs = [m.Job(0, 0, 700, 11, "pencil"), m.Job(1, 1, 900, 22, "uniform"),
            m.Job(0, 0, 0, 33, "uniform"), m.Job(1, 1, 500, 44, "uniform", 7)]
    _compare([g1, g2], [p1, p2], jobs, table)


def test_ragged_grids(table):
    """a one-voxel grid (every photon on the lateral mirrors, the bottom voxel
    continued below by the clamp addressing) and a one-voxel-high slab with three
    different voxel sizes, in one launch"""
    p = m.OpticalProps.from_tissues([(0.5, 10.0, 0.9, 1.4)])
    g1 = m.Geometry(np.ones((1, 1, 1), np.uint8), 0.1, 0.1, 0.1)
    g2 = m.Geometry(np.ones((5, 1, 7), np.uint8), 0.05, 0.2, 0.13)
    r = _compare([g1, g2], [p], [m.Job(0, 0, 2000, 8080, "uniform"),
                                 m.Job(1, 0, 2000, 9090, "pencil")], table)
    assert r[0].totals["quickfix"] > 0 and r[0].totals["r_in"] > 0
    for g, rr, beam in ((g1, r[0], "uniform"), (g2, r[1], "pencil")):
        fast = m.run([g], [p], [m.Job(0, 0, 20000, 77, beam)], table=table)[0]
        assert residual(fast.totals) == 0 and fast.totals["photons"] == 20000


def test_many_tissue_types(table):
    """250 tissue types with random refractive indices in random voxels: Fresnel at
    almost every face, optical-table lines up to the largest tissue index"""
    rng = np.random.default_rng(250)
    rows = [(rng.uniform(0.05, 1.0), rng.uniform(5, 20), rng.uniform(0.7, 0.95),
             rng.uniform(1.33, 1.5)) for _ in range(250)]
    g = m.Geometry(rng.integers(1, 251, (9, 10, 12)).astype(np.uint8), 0.1, 0.1, 0.1)
    p = m.OpticalProps.from_tissues(rows)
    r = _compare([g], [p], [m.Job(0, 0, 3000, 2501, "uniform")], table)
    assert r[0].totals["fresnel"] > 50 * r[0].totals["photons"]
    fast = m.run([g], [p], [m.Job(0, 0, 20000, 2502, "uniform")], table=table)[0]
    assert residual(fast.totals) == 0 and fast.totals["photons"] == 20000


def test_absorption_map(table):
    """the per-voxel absorbed weight (the reference's disabled tally,
    src/mc3d_gpu.cu:265-272) matches the oracle voxel for voxel and sums exactly to
    the absorbed total; enabling it changes no other tally"""
    g, p = layered(40, 36, 24, 0.1, air_holes=True)
    job = m.Job(0, 0, 2500, 97531, "uniform")
    r = m.run([g], [p], [job], table=table, math="exact", absorption_map=True)[0]
    o = oracle_job(g, p, job, table, absorption_map=True)
    assert np.array_equal(r.absorption, o["absorption"])
    assert int(r.absorption.sum()) == r.totals["absorbed"]
    plain = m.run([g], [p], [job], table=table, math="exact")[0]
    assert plain.totals == r.totals and np.array_equal(plain.drs, r.drs)
    fast = m.run([g], [p], [job], table=table, absorption_map=True)[0]
    assert int(fast.absorption.sum()) == fast.totals["absorbed"]
