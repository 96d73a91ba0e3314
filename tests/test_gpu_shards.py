"""The engine's multi-GPU data path on one GPU.

A job split into RNG-stream shards (Job.stream_first / stream_count) runs the same
photons with the same generators as the whole job, so the shards' integer tallies
add up to the whole job's bit for bit.  The first tests run the shards through
mc3d_run; the last runs them in two gloo ranks, each driving the engine on cuda:0,
and merges them with shard.all_reduce_results, the exchange bench.py uses over
NCCL.  The ranks' kernels are independent (no kernel waits on another rank), so
sharing one GPU is safe.  The seeding the shards partition is the reference's
per-slot init_RNG (src/mc3d_gpu.cu:454-455).
"""
from __future__ import annotations

import os
import random
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _case():
    import ymc3d_b200 as m
    from ymc3d_b200.workloads import LAYER_ROWS, layered_vessel_geometry
    g = layered_vessel_geometry(48, 40, 24, 0.1)
    p = m.OpticalProps.from_tissues(LAYER_ROWS)
    return g, p, m.Job(0, 0, 200_000, 8642, "uniform")


def _sum(parts):
    import ymc3d_b200 as m
    drs = sum(r.drs for r in parts)
    sq = sum(r.drs_sq for r in parts)
    tr = sum(r.trans for r in parts)
    tot = {k: sum(r.totals[k] for r in parts) for k in m.TOTAL_FIELDS}
    return drs, sq, tr, tot


@pytest.mark.parametrize("world,steps", [(2, "merged"), (3, "merged"), (3, "voxel")])
def test_shards_sum_to_whole_job(engine, table, world, steps):
    from ymc3d_b200.shard import shard_job
    g, p, job = _case()
    whole = engine.run([g], [p], [job], table=table, steps=steps)[0]
    parts = [engine.run([g], [p], [shard_job(job, r, world)], table=table, steps=steps)[0]
             for r in range(world)]
    assert all(0 < r.photons < job.photons for r in parts)
    drs, sq, tr, tot = _sum(parts)
    assert tot == whole.totals
    assert np.array_equal(drs, whole.drs) and np.array_equal(sq, whole.drs_sq)
    assert np.array_equal(tr, whole.trans)


def test_shards_in_one_launch(engine, table):
    """the shards as jobs of one batched launch, summed, equal the whole job"""
    from ymc3d_b200.shard import shard_job
    g, p, job = _case()
    whole = engine.run([g], [p], [job], table=table)[0]
    parts = engine.run([g], [p], [shard_job(job, r, 4) for r in range(4)], table=table)
    drs, sq, tr, tot = _sum(parts)
    assert tot == whole.totals and np.array_equal(drs, whole.drs)
    assert np.array_equal(sq, whole.drs_sq) and np.array_equal(tr, whole.trans)


def _worker(rank, world, port, tab, out):
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    import ymc3d_b200 as m
    from ymc3d_b200.shard import all_reduce_results, shard_job
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        g, p, job = _case()
        mine = m.run([g], [p], [shard_job(job, rank, world)], table=tab, device=0)
        merged = all_reduce_results(mine)[0]
        if rank == 0:
            out.put((merged.drs.copy(), merged.drs_sq.copy(), merged.trans.copy(),
                     merged.totals))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gloo_ranks_run_the_engine(engine, table):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    tab = np.asarray(table)
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, tab, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    try:
        drs, sq, tr, totals = q.get(timeout=300)
    finally:
        for pr in procs:
            pr.join(timeout=120)
    assert all(pr.exitcode == 0 for pr in procs)
    g, p, job = _case()
    whole = engine.run([g], [p], [job], table=table)[0]
    assert totals == whole.totals
    assert np.array_equal(drs, whole.drs) and np.array_equal(sq, whole.drs_sq)
    assert np.array_equal(tr, whole.trans)
