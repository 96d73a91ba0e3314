"""Splitting one job over ranks and merging the ranks' tallies.

Photons are independent, and stream i of a job always runs the same photons with
the same generator, so rank r of W can run the stream range shard_range(S, r, W)
of the job (Job.stream_first / stream_count) and the sum of the ranks' integer
tallies is bit-identical to a one-GPU run of the whole job.  The sum is the path's
only exchange: one all-reduce of (3 nx ny + 14) int64 words per step, over NCCL
between GPUs or gloo on CPU.
"""
from __future__ import annotations

import numpy as np

from . import TOTAL_FIELDS, Job, Result


def shard_range(streams: int, rank: int, world: int) -> tuple[int, int]:
    """[first, first + count) of `streams` owned by `rank` (contiguous, balanced)."""
    first = rank * streams // world
    return first, (rank + 1) * streams // world - first


def shard_job(job: Job, rank: int, world: int) -> Job:
    S = job.num_streams()
    first, count = shard_range(S, rank, world)
    return Job(job.geom, job.props, job.photons, job.seed, job.beam, S, stream_first=first,
               stream_count=count)


def pack(results: list[Result]) -> np.ndarray:
    parts = []
    for r in results:
        parts += [r.drs.reshape(-1), r.drs_sq.reshape(-1), r.trans.reshape(-1),
                  np.array([r.totals[k] for k in TOTAL_FIELDS], np.uint64)]
    return np.concatenate(parts).view(np.int64)


def unpack(flat: np.ndarray, like: list[Result]) -> list[Result]:
    a = flat.view(np.uint64)
    out, off = [], 0
    for r in like:
        nb = r.drs.size
        drs = a[off: off + nb].reshape(r.drs.shape).copy(); off += nb
        sq = a[off: off + nb].reshape(r.drs.shape).copy(); off += nb
        tr = a[off: off + nb].reshape(r.drs.shape).copy(); off += nb
        tot = {k: int(v) for k, v in zip(TOTAL_FIELDS, a[off: off + len(TOTAL_FIELDS)])}
        off += len(TOTAL_FIELDS)
        out.append(Result(drs, sq, tr, tot))
    return out


def all_reduce_results(results: list[Result], group=None, device=None) -> list[Result]:
    """Sum every rank's tallies (uint64 wrap-around arithmetic, exact) with
    torch.distributed; `device` is the CUDA device for NCCL, None for gloo."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(pack(results).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return unpack(t.cpu().numpy(), results)
