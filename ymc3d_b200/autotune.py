"""Launch-shape autotuner for photon-tracking plans.

Tallies do not depend on the launch shape (streams, not threads, own the random
numbers), so the shape is a pure speed choice.  The tuner runs a sample of the
real jobs -- the first streams of each -- under each candidate (threads per
block, blocks per SM), times it with CUDA events and keeps the fastest.  Choices
are cached per (device name, workload signature) in memory and in
_data/tuning.json next to the library.
"""
from __future__ import annotations

import hashlib
import json
import os
import time

from . import HERE, Job, Plan, default_table

# (threads per block, blocks per SM; 0 = as many as fit).  The photon kernels are
# built for 80 registers, so an SM holds 768 of their threads: 3 blocks of 256 or 6
# of 128 fill it (24 warps); 2 of 256 or 4 of 128 hold 16 warps, fewer to hide
# latency with.  Each block holds 28 KB of per-thread tally columns sized for 256
# threads, so blocks below 128 threads run out of shared memory before they fill
# an SM.
CANDIDATES = ((256, 0), (128, 0), (256, 2), (128, 4))
_CACHE_FILE = HERE / "_data" / "tuning.json"
_cache: dict | None = None


def _load() -> dict:
    global _cache
    if _cache is None:
        try:
            _cache = json.loads(_CACHE_FILE.read_text())
        except Exception:
            _cache = {}
    return _cache


def _save() -> None:
    try:
        _CACHE_FILE.parent.mkdir(exist_ok=True)
        tmp = _CACHE_FILE.with_suffix(f".tmp{os.getpid()}")
        tmp.write_text(json.dumps(_cache, indent=1, sort_keys=True))
        os.replace(tmp, _CACHE_FILE)
    except Exception:
        pass


def signature(geoms, props, jobs, math: str, steps: str = "merged") -> str:
    h = hashlib.sha1()
    for g in geoms:
        h.update(repr((g.shape, g.dx, g.dy, g.dz)).encode())
        h.update(hashlib.sha1(g.tissue.tobytes()).digest())
    for p in props:
        h.update(p.mua.tobytes() + p.mus.tobytes() + p.g.tobytes() + p.n.tobytes())
    for j in jobs:
        h.update(repr((j.geom, j.props, j.beam, int(j.photons) // 1000)).encode())
    h.update(math.encode())
    h.update(steps.encode())
    return h.hexdigest()[:16]


def _sample_jobs(jobs, streams_per_job: int):
    out = []
    for j in jobs:
        S = j.num_streams()
        out.append(Job(j.geom, j.props, j.photons, j.seed, j.beam, S, stream_first=0,
                       stream_count=min(S, streams_per_job)))
    return out


def tune(geoms, props, jobs, table=None, math: str = "fast", device: int = 0,
         candidates=CANDIDATES, sample_streams: int = 0, reps: int = 2,
         use_cache: bool = True, steps: str = "merged") -> dict:
    """Return {"block", "blocks_per_sm", "ms", "table"} for the fastest candidate."""
    import torch

    dev_name = torch.cuda.get_device_name(device)
    key = f"{dev_name}|{signature(geoms, props, jobs, math, steps)}"
    cache = _load()
    if use_cache and key in cache:
        return cache[key]
    table = default_table() if table is None else table
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    if not sample_streams:
        # sixteen streams per thread of a full grid (768 threads per SM), shared by the
        # jobs: a launch's tail is about one photon per thread, and it favours fewer
        # threads, so a short sample would pick shapes that lose in the steady state
        sample_streams = max(1, (sms * 768 * 16) // max(1, len(jobs)))
    sample = _sample_jobs(jobs, sample_streams)
    stream = torch.cuda.Stream(device)
    results = []
    for block, bps in candidates:
        try:
            plan = Plan(geoms, props, sample, table=table, math=math, device=device, block=block,
                        blocks_per_sm=bps, steps=steps)
        except Exception:
            continue
        plan.execute(stream.cuda_stream)
        stream.synchronize()
        times = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.execute(stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        results.append({"block": block, "blocks_per_sm": bps, "ms": min(times),
                        "grid": plan.shape()[1]})
        plan.close()
    if not results:
        raise RuntimeError("no launch shape could be planned")
    best = min(results, key=lambda r: r["ms"])
    choice = {"block": best["block"], "blocks_per_sm": best["blocks_per_sm"], "ms": best["ms"],
              "table": results, "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    cache[key] = choice
    _save()
    return choice
