"""Two gloo ranks on CPU: a job split into stream shards, each shard simulated by
the oracle, the shards' tallies summed with all_reduce -- bit-identical to the
whole job.  This is the engine's multi-GPU data path with the GPU run replaced
by its checker."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _job():
    import ymc3d_b200 as m
    g = m.Geometry(np.ones((16, 16, 16), np.uint8), 0.1, 0.1, 0.1)
    p = m.OpticalProps.from_tissues([(0.1, 10.0, 0.9, 1.4)])
    return g, p, m.Job(0, 0, 1500, 24680, "uniform", 333)


def _oracle_result(job, table, first, count):
    import oracle
    import ymc3d_b200 as m
    g, p, _ = _job()
    o = oracle.run(g.tissue, g.dx, g.dy, g.dz, p.mua, p.mus, p.g, p.n, job.photons,
                   job.num_streams(), job.seed, table, beam=m.BEAMS[job.beam], threads=1,
                   first=first, count=count)
    return m.Result(o["drs"], o["drs_sq"], o["trans"], o["totals"])


def _worker(rank, world, port, table, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    from ymc3d_b200.shard import all_reduce_results, shard_job
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    _, _, job = _job()
    sj = shard_job(job, rank, world)
    mine = _oracle_result(job, table, sj.stream_first, sj.stream_count)
    merged = all_reduce_results([mine])[0]
    if rank == 0:
        out.put((merged.drs.copy(), merged.trans.copy(), merged.totals))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_job_equals_whole_job(orc, table, world):
    import random
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    tab = np.asarray(table[:5000])
    procs = [ctx.Process(target=_worker, args=(r, world, port, tab, q)) for r in range(world)]
    for p in procs:
        p.start()
    drs, trans, totals = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    _, _, job = _job()
    whole = _oracle_result(job, tab, 0, -1)
    assert totals == whole.totals
    assert np.array_equal(drs, whole.drs) and np.array_equal(trans, whole.trans)


def test_shard_ranges_cover_streams():
    from ymc3d_b200.shard import shard_range
    for S in (1, 7, 1000, 4194304):
        for W in (1, 2, 3, 8):
            got = [shard_range(S, r, W) for r in range(W)]
            assert got[0][0] == 0 and sum(c for _, c in got) == S
            assert all(got[i][0] + got[i][1] == got[i + 1][0] for i in range(W - 1))
