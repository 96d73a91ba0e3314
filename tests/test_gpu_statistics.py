"""Fast-math kernel: statistical parity, exact conservation and bit-reproducible
tallies across launch shapes and batching."""
from __future__ import annotations

import numpy as np
import pytest

import ymc3d_b200 as m
from helpers import drs_chi2, oracle_job, residual, total_z

pytestmark = pytest.mark.gpu


def layered_small():
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    return layered_vessel_geometry(64, 64, 32, 0.08), m.OpticalProps.from_tissues(LAYER_ROWS)


def test_fast_vs_exact_chi2(table):
    g, p = layered_small()
    fast = m.run([g], [p], [m.Job(0, 0, 2_000_000, 5, "uniform")], table=table, math="fast")[0]
    exact = m.run([g], [p], [m.Job(0, 0, 2_000_000, 6, "uniform")], table=table,
                  math="exact")[0]
    chi2, dof, pv = drs_chi2(fast.drs, fast.drs_sq, fast.photons, exact.drs, exact.drs_sq,
                             exact.photons, f=8)
    assert dof > 20 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "absorbed"):
        assert abs(total_z(fast.totals, exact.totals, key)) < 5


def test_fast_vs_exact_pencil_chi2(table):
    """pencil beam into a homogeneous slab: the radial fall-off of the DRS is steep,
    so a bias of the fast path's crossing logic would show in the inner bins"""
    g = m.Geometry(np.ones((48, 64, 64), np.uint8), 0.05, 0.05, 0.05)
    p = m.OpticalProps.from_tissues([(0.02, 8.0, 0.9, 1.37)])
    fast = m.run([g], [p], [m.Job(0, 0, 3_000_000, 11, "pencil")], table=table)[0]
    exact = m.run([g], [p], [m.Job(0, 0, 3_000_000, 12, "pencil")], table=table,
                  math="exact")[0]
    chi2, dof, pv = drs_chi2(fast.drs, fast.drs_sq, fast.photons, exact.drs, exact.drs_sq,
                             exact.photons, f=2)
    assert dof > 100 and pv > 1e-4, (chi2, dof, pv)
    for key in ("r_in", "r_out", "absorbed"):
        assert abs(total_z(fast.totals, exact.totals, key)) < 5, key


def test_fast_vs_oracle_chi2(table):
    g, p = m.Geometry(np.ones((32, 32, 32), np.uint8), 0.1, 0.1, 0.1), \
        m.OpticalProps.from_tissues([(0.05, 10.0, 0.9, 1.4)])
    job = m.Job(0, 0, 40_000, 2024, "pencil")
    fast = m.run([g], [p], [job], table=table, math="fast")[0]
    o = oracle_job(g, p, m.Job(0, 0, 40_000, 2025, "pencil"), table)
    chi2, dof, pv = drs_chi2(fast.drs, fast.drs_sq, fast.photons, o["drs"], o["drs_sq"],
                             o["totals"]["photons"], f=4)
    assert dof > 10 and pv > 1e-4, (chi2, dof, pv)
    assert abs(total_z(fast.totals, o["totals"], "r_in")) < 5


def test_conservation_exact(table):
    g, p = layered_small()
    r = m.run([g], [p], [m.Job(0, 0, 1_000_000, 77, "uniform")], table=table)[0]
    t = r.totals
    assert t["photons"] == 1_000_000
    assert residual(t) == 0
    assert int(r.drs.sum()) == t["r_in"]
    assert int(r.trans.sum()) == t["t_in"]
    assert t["w_launched"] > 0 and t["steps"] > t["photons"]


@pytest.mark.parametrize("block,bps", [(64, 1), (128, 3), (256, 0), (96, 2), (256, 4),
                                       (128, 8)])
def test_launch_shape_reproducible(table, block, bps):
    g, p = layered_small()
    job = m.Job(0, 0, 300_000, 4242, "uniform")
    base = m.run([g], [p], [job], table=table)[0]
    r = m.run([g], [p], [job], table=table, block=block, blocks_per_sm=bps)[0]
    assert r.totals == base.totals
    assert np.array_equal(r.drs, base.drs) and np.array_equal(r.drs_sq, base.drs_sq)


def test_batched_equals_separate(table):
    from ymc3d_b200.workloads import sweep
    w = sweep(njobs=6, photons_lo=2e4, photons_hi=2e5)
    together = m.run(w.geoms, w.props, w.jobs, table=table)
    for job, r in zip(w.jobs, together):
        alone = m.run(w.geoms, [w.props[job.props]], [m.Job(0, 0, job.photons, job.seed,
                                                             job.beam)], table=table)[0]
        assert r.totals == alone.totals
        assert np.array_equal(r.drs, alone.drs)


def test_many_geometries_batched_equals_separate(table):
    """64 geometries in one launch (descriptors and tables in shared memory,
    with the tally columns over 48 KB per block): each job's tallies equal its
    run alone"""
    from ymc3d_b200.workloads import uneven
    w = uneven(ngeoms=64, photons=10_000, max_dim=72)
    assert sum(3 * 16 * p.num_tissue_types for p in w.props) + 64 * 72 + 28672 > 48 * 1024
    together = m.run(w.geoms, w.props, w.jobs, table=table)
    for k in (0, 17, 63):
        job = w.jobs[k]
        alone = m.run([w.geoms[job.geom]], [w.props[job.props]],
                      [m.Job(0, 0, job.photons, job.seed, job.beam)], table=table)[0]
        assert together[k].totals == alone.totals
        assert np.array_equal(together[k].drs, alone.drs)


def test_plan_reexecute_identical(table):
    g, p = layered_small()
    plan = m.Plan([g], [p], [m.Job(0, 0, 200_000, 9, "uniform")], table=table)
    plan.execute()
    a = plan.read()[0]
    plan.execute()
    b = plan.read()[0]
    plan.close()
    assert a.totals == b.totals and np.array_equal(a.drs, b.drs)


def test_plan_memory_returns_to_the_pool(table):
    """plans take device memory from the library's pool and give it back: after
    the first plan, creating and destroying more (merged-step maps, absorption
    map, graph capture, mc3d_run) leaves the device's free memory where it was,
    and a plan built after many others still gives the same tallies"""
    import torch
    g, p = layered_small()
    jobs = [m.Job(0, 0, 50_000, 9, "uniform")]
    first = m.run([g], [p], jobs, table=table)[0]
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    for k in range(12):
        plan = m.Plan([g], [p], jobs, table=table, use_graph=(k % 2 == 1))
        plan.execute()
        plan.read()
        plan.close()
        m.run([g], [p], jobs, table=table, absorption_map=(k % 3 == 0))
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free1 >= free0 - (64 << 20), (free0, free1)
    again = m.run([g], [p], jobs, table=table)[0]
    assert again.totals == first.totals and np.array_equal(again.drs, first.drs)


def test_plan_graph_replay_identical(table):
    """a plan captured into a CUDA graph replays to the same tallies"""
    g, p = layered_small()
    jobs = [m.Job(0, 0, 150_000, 9, "uniform"), m.Job(0, 0, 50_000, 10, "pencil")]
    direct = m.run([g], [p], jobs, table=table)
    plan = m.Plan([g], [p], jobs, table=table, use_graph=True)
    for _ in range(3):
        plan.execute()
        got = plan.read()
        for a, b in zip(got, direct):
            assert a.totals == b.totals and np.array_equal(a.drs, b.drs)
    plan.close()


def test_autotune_picks_a_shape_and_results_stay(table):
    from ymc3d_b200 import autotune
    g, p = layered_small()
    jobs = [m.Job(0, 0, 400_000, 31, "uniform")]
    choice = autotune.tune([g], [p], jobs, table=table, use_cache=False,
                           candidates=((256, 0), (128, 0), (64, 2)))
    assert choice["block"] in (256, 128, 64) and len(choice["table"]) == 3
    a = m.run([g], [p], jobs, table=table)[0]
    b = m.run([g], [p], jobs, table=table, block=choice["block"],
              blocks_per_sm=choice["blocks_per_sm"])[0]
    assert a.totals == b.totals and np.array_equal(a.drs, b.drs)


def test_cancel_flag_stops_and_keeps_partial_tallies_consistent(table):
    """the host-side stop (the reference stops on SIGINT, src/mc3d_gpu.cu:379-394,
    573-577): a flag set before the launch makes every thread stop at its first
    stream; the call reports MC3D_ERR_CANCELLED and the partial tallies still
    conserve weight exactly"""
    g, p = layered_small()
    flag = np.array([1], np.int32)
    with pytest.raises(m.Mc3dError) as e:
        m.run([g], [p], [m.Job(0, 0, 500_000, 3, "uniform")], table=table, cancel=flag)
    assert e.value.status == -12
    part = e.value.results[0]
    assert part.photons < 500_000
    assert part.conservation_residual() == 0


def test_skin_model_runs(table):
    """the MATLAB example model, restated in workloads.py, through the engine:
    exact conservation and reflectance from every layer's surface bins"""
    from ymc3d_b200 import workloads as W
    g = W.skin_geometry()
    p = W.skin_optprops(600.0, lambda oxy, lam: 2e4 * (1 + oxy))
    r = m.run([g], [p], [m.Job(0, 0, 200_000, 5, "uniform")], table=table)[0]
    assert r.photons == 200_000 and residual(r.totals) == 0
    assert 0 < r.totals["r_in"] < r.totals["w_launched"]


@pytest.mark.parametrize("which", ["layered", "deep"])
def test_full_size_invariants(table, which):
    """the benchmark's full sizes, through size-independent properties: the
    layered 256x256x128 job at 1e8 photons and the 1024x1024x256 grid (256 MB,
    beyond L2) at 1e7 conserve weight exactly, their bins sum to the totals, and
    every photon finishes (none at the step cap)"""
    from ymc3d_b200.workloads import deep_grid, layered_vessel
    w = layered_vessel(photons=100_000_000) if which == "layered" else deep_grid(photons=10_000_000)
    r = m.run(w.geoms, w.props, w.jobs, table=table)[0]
    t = r.totals
    assert t["photons"] == w.jobs[0].photons and residual(t) == 0
    assert int(r.drs.sum()) == t["r_in"] and int(r.trans.sum()) == t["t_in"]
    assert t["capped"] == 0
