"""Benchmark: photons/s of the photon-tracking path on B200.

Workload: the layered tissue with a vessel, 256x256x128 voxels of 0.02 mm, uniform
beam, a job of 1e8 photons per GPU; one step is one launch of the whole job.

  value  device throughput: photons / kernel time, inputs resident in HBM, timed
         with CUDA events on the launching stream, L2 flushed between steps.
  e2e    the same through the C ABI from pinned host buffers (mc3d_run: geometry,
         optical table and safe-prime table uploaded, tallies read back each step),
         timed on the host around the synchronous call.

--impl reference runs the reference's own run_3dmc_gpu (compiled from its sources
into oracle/_ref/gpu-mc-ref) on the same workload and GPU, on a bounded photon
sample.  With torchrun (--gpus N) every rank runs one shard of a job of
N x photons (disjoint RNG streams, weak scaling); the shards' integer tallies are
summed over NCCL once per step, which is the path's only exchange.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

# Algorithmic operations per photon step, counted from the reference formulas
# (src/mc3d_gpu.cu:181-339; each +, -, *, /, comparison, min, sqrt, rsqrt, log,
# sin/cos counted once, integer and select operations not counted).  Of the 152,
# 20 are special-function class (13 divisions, 2 sqrt, 2 rsqrt, 1 log, sin+cos of
# sincospif); a Fresnel event (:226-257) adds 37, 6 of them special (acos, sin,
# sqrt, 3 divisions).
OPS_STEP, SFU_STEP = 152, 20
# a merged step adds the jump: radius x unit, compare, 3 x (x + u R)
OPS_JUMP = 8
OPS_FRESNEL, SFU_FRESNEL = 37, 6
FP32_LANES_PER_SM, SFU_LANES_PER_SM = 128, 16
# DRAM bytes read + written by one photon-kernel launch of the layered workload
# (ncu dram__bytes_read.sum + dram__bytes_write.sum = 30,852,096 + 0 on a
# 1e7-photon launch): the first touch of grid, packed cell map, table and tallies,
# independent of the photon count
TRAFFIC_BYTES_PER_LAUNCH = 30_852_096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--photons", type=float, default=1e8, help="photons per GPU per job")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--math", default="fast", choices=["fast", "exact", "f64"])
    ap.add_argument("--ref-photons", type=float, default=1e7)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the launch-shape autotuner")
    ap.add_argument("--step-mode", default="merged", choices=["merged", "voxel"],
                    help="fast math: merged crossings in uniform tissue, or one step per voxel face")
    ap.add_argument("--workload", default="layered",
                    choices=["layered", "homogeneous", "sweep", "uneven", "deep", "precision"],
                    help="layered is the headline; the others are the batched and "
                         "special configurations, one launch per step")
    ap.add_argument("--beam", default="uniform", choices=["uniform", "pencil"],
                    help="beam of the sweep workload (the reference has only uniform)")
    ap.add_argument("--photon-scale", type=float, default=0.01,
                    help="photon budget factor of the sweep / uneven / deep workloads")
    ap.add_argument("--sweep-scale", type=float, default=1.0,
                    help="photon budget factor of the sweep object of the default run")
    ap.add_argument("--no-sweep", action="store_true",
                    help="leave the sweep object out of the default run")
    ap.add_argument("--sweep-ref-seconds", type=float, default=30.0,
                    help="reference arm: time budget per sampled sweep job (its four seeded "
                         "calls, whose batch means give sigma)")
    ap.add_argument("--ref-warmup-photons", type=float, default=230400,
                    help="reference arm: photons of each warm-up call (the slot count)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.out,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.out.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "samples": len(sm),
                "reasons": sorted(reasons)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {"sm_max_mhz": 1965.0, "fallback": True}


def cpu_baseline(w, seconds: float) -> dict:
    """The oracle (scalar C, OpenMP over streams) on the first streams of the same job."""
    import oracle
    from ymc3d_b200 import default_table
    g, p, job = w.geoms[0], w.props[0], w.jobs[0]
    table = default_table()
    cores = os.cpu_count() or 1
    S = job.num_streams()
    count = max(cores * 4, 64)
    while True:
        t0 = time.perf_counter()
        r = oracle.run(g.tissue, g.dx, g.dy, g.dz, p.mua, p.mus, p.g, p.n, int(job.photons), S,
                       int(job.seed), table, beam=0, threads=cores, first=0, count=count)
        dt = time.perf_counter() - t0
        if dt > seconds / 4 or count * (job.photons // S) >= 5_000_000:
            break
        count = int(count * min(8.0, max(2.0, seconds / 2 / max(dt, 1e-3))))
    nph = r["totals"]["photons"]
    return {"value": nph / dt, "unit": "photons/s", "cores": cores, "kind": "port",
            "sample": f"{nph} photons (first {count} RNG streams of the same job), "
                      f"{r['totals']['steps']} steps, {dt:.2f} s",
            "steps_per_s": r["totals"]["steps"] / dt}


def run_ours(args):
    import torch

    import ymc3d_b200 as m
    from ymc3d_b200.shard import all_reduce_results
    from ymc3d_b200.workloads import layered_vessel

    world, rank, local, dist = dist_setup(args)
    dev = local
    torch.cuda.set_device(dev)
    per_gpu = int(args.photons)
    w = layered_vessel(photons=per_gpu * world)
    job = w.jobs[0]
    S = job.num_streams()

    def shard(j: "m.Job") -> "m.Job":
        """this rank's stream range of job j"""
        Sj = j.num_streams()
        first = rank * Sj // world
        return m.Job(j.geom, j.props, j.photons, j.seed, j.beam, Sj, stream_first=first,
                     stream_count=(rank + 1) * Sj // world - first)

    g = w.geoms[0]
    pinned = torch.empty(g.tissue.size, dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = g.tissue.reshape(-1)
    geom = m.Geometry(pinned.numpy().reshape(g.tissue.shape), g.dx, g.dy, g.dz)
    table = m.default_table()
    pinned_tab = torch.empty(len(table), dtype=torch.int32, pin_memory=True)
    pinned_tab.numpy().view(np.uint32)[:] = table
    table_p = pinned_tab.numpy().view(np.uint32)
    # warm-up job: the same workload at a tenth of the photons, another seed
    warm_job = m.Job(job.geom, job.props, max(1, job.photons // 10), job.seed + 1, job.beam)

    tuned = {"block": 0, "blocks_per_sm": 0, "table": []}
    if not args.no_tune:
        from ymc3d_b200 import autotune
        tuned = autotune.tune([geom], w.props, [shard(warm_job)], table=table_p, math=args.math,
                              device=dev, use_cache=False, steps=args.step_mode)
    shape = {"block": tuned["block"], "blocks_per_sm": tuned["blocks_per_sm"],
             "steps": args.step_mode}
    plan = m.Plan([geom], w.props, [shard(job)], table=table_p, math=args.math, device=dev,
                  **shape)
    warm_plan = m.Plan([geom], w.props, [shard(warm_job)], table=table_p, math=args.math,
                       device=dev, **shape)
    stream = torch.cuda.Stream(dev)  # a real stream handle (the legacy default stream is 0)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    nb = g.tissue.shape[1] * g.tissue.shape[2]

    def exchange(res):
        """sum the shards' integer tallies over NCCL (the path's exchange step)"""
        if world == 1:
            return res
        return all_reduce_results(res, device=torch.device("cuda", dev))

    for k in range(args.warmup):
        warm_plan.execute(stream.cuda_stream)
        exchange(warm_plan.read())
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    times, steps_tot, fresnel_tot, photons_tot = [], 0, 0, 0
    launches = 0
    with ClockSampler(dev) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xff)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.execute(stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            launches += 1
            times.append(e0.elapsed_time(e1) / 1e3)
            res = exchange(plan.read())
            steps_tot += res[0].totals["steps"]
            fresnel_tot += res[0].totals["fresnel"]
            photons_tot += res[0].totals["photons"]
    torch.cuda.synchronize(dev)
    t_step = sum(times) / len(times)
    if dist:
        tt = torch.tensor([t_step], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_step = float(tt.item())
    photons_step = photons_tot / args.steps  # whole job after the exchange
    value = photons_step / t_step

    e2e = None
    if not args.no_e2e:
        e2e_times = []
        h2d = g.tissue.size + table_p.nbytes + sum(p.mua.nbytes * 4 for p in w.props)
        d2h = 3 * nb * 8 + 14 * 8
        e2e_photons = 0
        # one untimed call through the same API first: the first mc3d_run of a
        # process pays one-time driver costs (about 1 s measured)
        exchange(m.run([geom], w.props, [shard(warm_job)], table=table_p, math=args.math,
                       device=dev, **shape))
        for k in range(max(1, args.e2e_steps)):
            flush.fill_(k & 0xff)
            torch.cuda.synchronize(dev)
            if dist:
                dist.barrier()
            t0 = time.perf_counter()
            res = m.run([geom], w.props, [shard(job)], table=table_p, math=args.math, device=dev,
                        **shape)
            res = exchange(res)
            e2e_times.append(time.perf_counter() - t0)
            e2e_photons += res[0].totals["photons"]
        te = sum(e2e_times) / len(e2e_times)
        if dist:
            tt = torch.tensor([te], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            te = float(tt.item())
        e2e = {"value": e2e_photons / len(e2e_times) / te, "unit": "photons/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": te * 1e3,
               "samples_ms": [round(t * 1e3, 1) for t in e2e_times],
               "warmup": "one untimed mc3d_run of the warm-up job",
               "timing": "host clock around the synchronous mc3d_run call (plan, upload, "
                         "kernel, read-back), max over ranks"}

    if rank != 0:
        plan.close()
        warm_plan.close()
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    pk = peaks()
    clk = clocks.summary()
    f_max = float(pk.get("sm_max_mhz", 1965.0)) * 1e6
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    steps_per_s = steps_tot / args.steps / world / t_step  # per GPU
    fres_per_s = fresnel_tot / args.steps / world / t_step
    sfu_ops = steps_per_s * SFU_STEP + fres_per_s * SFU_FRESNEL
    ops_step = OPS_STEP + (OPS_JUMP if args.math == "fast" and args.step_mode == "merged" else 0)
    fp32_ops = steps_per_s * (ops_step - SFU_STEP) + fres_per_s * (OPS_FRESNEL - SFU_FRESNEL)
    sfu_peak = sms * SFU_LANES_PER_SM * f_max
    fp32_peak = sms * FP32_LANES_PER_SM * f_max
    traffic = TRAFFIC_BYTES_PER_LAUNCH
    block, grid, smem = plan.shape()
    line = {
        "metric": "photons/s (layered tissue + vessel, 256x256x128, uniform beam, 1 B200)",
        "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64+u64" if args.math == "f64" else "f32+u64",
        "data": "synthetic (seeded layered-tissue geometry, reference input formats)",
        "config": {"workload": w.name, "photons_per_job": int(job.photons),
                   "photons_per_step": int(photons_step),
                   "step": "one launch of the whole job (each rank: its stream shard)",
                   "warmup": "3 launches of the same workload at a tenth of the photons", "voxels": list(g.shape), "voxel_mm": g.dx,
                   "beam": "uniform", "math": args.math, "step_mode": args.step_mode,
                   "streams": S,
                   "launch": {"block": block, "grid": grid, "smem": smem,
                              "autotuner": [{k: r[k] for k in ("block", "blocks_per_sm", "ms")}
                                            for r in tuned["table"]]},
                   "l2": "flushed between steps (256 MB write)",
                   "parallelism": f"{world} ranks, disjoint stream shards, NCCL sum of tallies"},
        "steps_per_s": steps_per_s * world,
        "roofline": {"bound": "sfu", "achieved": sfu_ops / 1e9, "peak": sfu_peak / 1e9,
                     "unit": "Gop/s", "frac": sfu_ops / sfu_peak, "traffic": traffic,
                     "peak_basis": f"{sms} SMs x {SFU_LANES_PER_SM} SFU lanes x sm_max "
                                   f"{f_max / 1e6:.0f} MHz (MEASURED_PEAKS.json clock)",
                     "fp32": {"achieved": fp32_ops / 1e9, "peak": fp32_peak / 1e9,
                              "frac": fp32_ops / fp32_peak},
                     "ops_per_step": {"all": ops_step, "sfu": SFU_STEP,
                                      "fresnel_all": OPS_FRESNEL, "fresnel_sfu": SFU_FRESNEL}},
        "clocks": clk,
        "gpu_launches": launches,  # one photon-kernel launch per step (after a tally memset)
        "e2e": e2e,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(w, args.cpu_seconds)
    plan.close()
    warm_plan.close()
    if world == 1 and not args.no_sweep:
        sw = measure_sweep(args, dev, stream, flush)
        sfu = (sw["_steps"] * SFU_STEP + sw["_fresnel"] * SFU_FRESNEL) / sw["_seconds"]
        sw["roofline"] = {"bound": "sfu", "achieved": sfu / 1e9, "peak": sfu_peak / 1e9,
                          "unit": "Gop/s", "frac": sfu / sfu_peak}
        for k in ("_steps", "_fresnel", "_seconds"):
            sw.pop(k)
        sw["gpu_launches"] = 1 + sw["jobs"]  # the batched launch, then one per job
        line["sweep"] = sw
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


SWEEP_STRATA = 8


def sweep_subset(w, strata: int = SWEEP_STRATA, seed: int = 20240611) -> list[int]:
    """A seeded stratified subset of the sweep's jobs for the reference arm: the jobs
    sorted by mua (which sets a photon's path length) in `strata` equal strata, one
    job drawn from each."""
    mua = np.array([float(w.props[j.props].mua[1]) for j in w.jobs])
    order = np.argsort(mua, kind="stable")
    rng = np.random.Generator(np.random.PCG64(seed))
    per = len(order) // strata
    return [int(order[s * per + int(rng.integers(per))]) for s in range(strata)]


def sweep_strata(w, strata: int = SWEEP_STRATA) -> list[list[int]]:
    mua = np.array([float(w.props[j.props].mua[1]) for j in w.jobs])
    order = np.argsort(mua, kind="stable")
    per = len(order) // strata
    return [[int(k) for k in order[s * per:(s + 1) * per]] for s in range(strata)]


def r_total_sigma(r) -> tuple[float, float]:
    """total diffuse reflectance per photon and its standard error; each photon's
    reflected weight lands in one bin, so the bins' sum W^2 is the photons' sum W^2"""
    n = max(1, r.photons)
    m1 = float(r.drs.sum()) / 4294967296.0 / n
    m2 = float(r.drs_sq.sum()) / 4294967296.0 / n
    return m1, float(np.sqrt(max(m2 - m1 * m1, 0.0) / n))


def measure_sweep(args, dev, stream, flush) -> dict:
    """The metric's own comparison on the hyperspectral sweep: 128 optical tables on
    the homogeneous 64^3 x 0.1 mm geometry, photons log-uniform in [1e6, 1e8] per
    job (2.75e9 in all at scale 1), uniform beam (the reference's only beam).
    Batched = one persistent launch over every job; plain = one launch per job with
    the same jobs and seeds.  Both give identical tallies (checked word for word),
    so their DRS sigma-errors are equal by construction."""
    import torch

    import ymc3d_b200 as m
    from ymc3d_b200 import workloads as W

    w = W.sweep(photon_scale=args.sweep_scale, beam="uniform")
    warm = W.sweep(photon_scale=1e-3, beam="uniform")
    wp = m.Plan(warm.geoms, warm.props, warm.jobs, device=dev, steps=args.step_mode)
    wp.execute(stream.cuda_stream)
    wp.read()
    wp.close()

    def timed(plan):
        flush.fill_(7)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    with ClockSampler(dev) as clocks:
        plan = m.Plan(w.geoms, w.props, w.jobs, device=dev, steps=args.step_mode)
        t_batch = timed(plan)
        batched = plan.read()
        plan.close()
        t_plain, identical = [], True
        for k, job in enumerate(w.jobs):
            pl = m.Plan([w.geoms[0]], [w.props[job.props]],
                        [m.Job(0, 0, job.photons, job.seed, job.beam)], device=dev,
                        steps=args.step_mode)
            t_plain.append(timed(pl))
            r = pl.read()[0]
            pl.close()
            b = batched[k]
            identical &= (r.totals == b.totals and np.array_equal(r.drs, b.drs)
                          and np.array_equal(r.drs_sq, b.drs_sq))
    photons = sum(r.photons for r in batched)
    steps = sum(r.totals["steps"] for r in batched)
    fresnel = sum(r.totals["fresnel"] for r in batched)
    rel = [sg / mu for mu, sg in map(r_total_sigma, batched) if mu > 0]
    sub = sweep_subset(w)
    return {"workload": w.name, "jobs": len(w.jobs), "photons": photons,
            "photon_scale": args.sweep_scale, "beam": "uniform", "step_mode": args.step_mode,
            "batched": {"value": photons / t_batch, "unit": "photons/s", "seconds": t_batch,
                        "how": "one persistent launch over all jobs (tally clear + kernel), "
                               "CUDA events, L2 flushed before"},
            "plain": {"value": photons / sum(t_plain), "unit": "photons/s",
                      "seconds": sum(t_plain),
                      "how": "one launch per job, same jobs and seeds, CUDA events summed, "
                             "L2 flushed before each"},
            "batched_over_plain": sum(t_plain) / t_batch,
            "tallies_identical": bool(identical),
            "sigma": {"r_total_rel_median": float(np.median(rel)),
                      "r_total_rel_max": float(np.max(rel)),
                      "how": "per job from sum W^2; batched and plain are identical, so "
                             "their sigma is equal"},
            "steps_per_s": steps / t_batch, "fresnel_per_s": fresnel / t_batch,
            "reference_subset": {
                "jobs": sub, "photons": int(sum(w.jobs[k].photons for k in sub)),
                "plain_seconds": float(sum(t_plain[k] for k in sub)),
                "r_total": [list(r_total_sigma(batched[k])) for k in sub],
                "how": "the jobs the reference arm runs (seeded, one per mua stratum); "
                       "this engine's plain time on them"},
            "clocks": clocks.summary(), "_steps": steps, "_fresnel": fresnel,
            "_seconds": t_batch}


def reference_sweep(args, exe: Path) -> dict:
    """The reference's run_3dmc_gpu on the stratified subset of the sweep.  Each
    sampled job runs as four seeded calls (batch means give its sigma): a pilot of
    230,400 photons (the reference's slot count and minimum), then three calls
    sized from the pilot's rate to fill --sweep-ref-seconds, never beyond the job's
    own photon count.  The reference's time for the whole sweep is estimated by
    strata: each stratum's photons times its sampled job's seconds per photon."""
    from ymc3d_b200 import workloads as W
    from ymc3d_b200.workloads import write_geometry_file, write_optprops_file
    w = W.sweep(photon_scale=args.sweep_scale, beam="uniform")
    sub = sweep_subset(w)
    strata = sweep_strata(w)
    tmp = Path(tempfile.mkdtemp())
    g = w.geoms[0]
    write_geometry_file(tmp / "geom.bin", g.tissue, g.dx, g.dy, g.dz)
    slots = 230_400

    def call(k, photons, seed, tag):
        out = tmp / f"s{k}_{tag}"
        subprocess.run([str(exe), str(tmp / "geom.bin"), str(tmp / f"p{k}.bid"), str(photons),
                        str(seed), str(out), str(exe.parent)], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        raw = Path(str(out) + "_ref.bin").read_bytes()
        fin = int(np.frombuffer(raw, "<i8", 1)[0])
        sec = float(np.frombuffer(raw, "<f8", 1, offset=8)[0])
        nx, ny = np.frombuffer(raw, "<i4", 2, offset=16)
        R = np.frombuffer(raw, "<f8", int(nx * ny), offset=24)
        return fin, sec, float(R.sum()) / fin

    jobs, t_est, fin_all, sec_all = [], 0.0, 0, 0.0
    for s_idx, k in enumerate(sub):
        job = w.jobs[k]
        p = w.props[job.props]
        write_optprops_file(tmp / f"p{k}.bid", np.stack([p.mua, p.mus, p.g, p.n], 1)[1:])
        seeds = [((int(job.seed) + 1000003 * b) & 0xFFFFFFFF) or 1 for b in range(4)]
        runs = [call(k, slots, seeds[0], 0)]
        rate = runs[0][0] / runs[0][1]
        left = max(0, int(job.photons) - runs[0][0])
        per = max(slots, min(left, int(rate * max(0.0, args.sweep_ref_seconds - runs[0][1])))
                  // 3)
        for b in (1, 2, 3):
            runs.append(call(k, per, seeds[b], b))
        fins = sum(r[0] for r in runs)
        secs = sum(r[1] for r in runs)
        rb = np.array([r[2] for r in runs])
        wts = np.array([r[0] for r in runs], float)
        mean = float(np.sum(rb * wts) / wts.sum())
        # batch means, weighted by each call's photons
        var = float(np.sum(wts * (rb - mean) ** 2) / wts.sum() / (len(rb) - 1))
        jobs.append({"job": k, "mua": float(p.mua[1]), "photons_of_job": int(job.photons),
                     "photons_run": fins, "calls": len(runs), "seconds": secs,
                     "value": fins / secs, "unit": "photons/s", "r_total": mean,
                     "r_total_sigma_batch_means": float(np.sqrt(var))})
        fin_all += fins
        sec_all += secs
        stratum_photons = sum(int(w.jobs[j].photons) for j in strata[s_idx])
        t_est += stratum_photons * secs / fins
    return {"workload": w.name, "jobs_total": len(w.jobs), "photons_total": w.photons,
            "photon_scale": args.sweep_scale, "beam": "uniform",
            "subset": {"jobs": jobs, "photons": fin_all, "seconds": sec_all,
                       "value": fin_all / sec_all, "unit": "photons/s",
                       "how": f"one seeded job per mua stratum ({SWEEP_STRATA} strata of "
                              f"{len(w.jobs) // SWEEP_STRATA}); four run_3dmc_gpu calls per "
                              "job (230,400 photons, then three sized to "
                              f"{args.sweep_ref_seconds:.0f} s in all, at most the job's "
                              "count); wall time of each call"},
            "full_sweep_estimate": {"seconds": t_est, "value": w.photons / t_est,
                                    "unit": "photons/s",
                                    "how": "each stratum's photons x its sampled job's "
                                           "seconds per finished photon"}}


def run_reference_batched(args, exe: Path):
    """The reference binary once per job of a batched workload (uniform beam: its
    pencil branch is compiled out), timed as the sum of its run_3dmc_gpu calls.
    The reference runs at least 230,400 photons per call (one per slot)."""
    from ymc3d_b200 import workloads as W
    from ymc3d_b200.workloads import write_geometry_file, write_optprops_file
    if args.workload == "sweep":
        w = W.sweep(photon_scale=args.photon_scale, beam="uniform")
    else:
        w = W.uneven(photons=max(1, int(1e7 * args.photon_scale)))
    tmp = Path(tempfile.mkdtemp())
    for gi, g in enumerate(w.geoms):
        write_geometry_file(tmp / f"geom{gi}.bin", g.tissue, g.dx, g.dy, g.dz)
    secs, fins = 0.0, 0
    for k, job in enumerate(w.jobs):
        p = w.props[job.props]
        rows = np.stack([p.mua, p.mus, p.g, p.n], 1)[1:]
        write_optprops_file(tmp / f"p{k}.bid", rows)
        subprocess.run([str(exe), str(tmp / f"geom{job.geom}.bin"), str(tmp / f"p{k}.bid"),
                        str(int(job.photons)), str(int(job.seed) & 0xffffffff or 1),
                        str(tmp / f"r{k}"), str(exe.parent)], check=True,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        raw = (tmp / f"r{k}_ref.bin").read_bytes()
        fins += int(np.frombuffer(raw, "<i8", 1)[0])
        secs += float(np.frombuffer(raw, "<f8", 1, offset=8)[0])
    line = {"metric": f"photons/s ({w.name}, uniform beam, 1 B200)", "value": fins / secs,
            "unit": "photons/s", "n_gpus": 1, "steps": 1, "warmup": 0,
            "ms_per_step": secs * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "jobs": len(w.jobs), "photons_per_step": fins,
                       "photon_scale": args.photon_scale,
                       "how": "one run_3dmc_gpu call per job, summed"},
            "impl": "reference"}
    print(json.dumps(line), flush=True)


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if args.workload in ("homogeneous", "precision", "deep"):
        why = {"homogeneous": "the workload's pencil beam is compiled out of the reference "
                              "(src/mc3d_gpu.cu:87-95)",
               "precision": "the reference has no FP64 stepping",
               "deep": "a 1e7-photon deep-grid run takes the reference minutes; its "
                       "per-photon cost is measured on the layered workload"}[args.workload]
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    if args.workload in ("sweep", "uneven"):
        exe = ROOT / "oracle" / "_ref" / "gpu-mc-ref"
        if not exe.exists():
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/gpu-mc-ref not built (oracle/build_ref.py)"}))
            return
        return run_reference_batched(args, exe)
    exe = ROOT / "oracle" / "_ref" / "gpu-mc-ref"
    if not exe.exists():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/gpu-mc-ref not built (oracle/build_ref.py)"}))
        return
    from ymc3d_b200.workloads import layered_vessel, write_geometry_file, write_optprops_file
    w = layered_vessel(photons=int(args.ref_photons))
    g = w.geoms[0]
    rows = np.stack([w.props[0].mua, w.props[0].mus, w.props[0].g, w.props[0].n], 1)[1:]
    tmp = Path(tempfile.mkdtemp())
    write_geometry_file(tmp / "geom.bin", g.tissue, g.dx, g.dy, g.dz)
    write_optprops_file(tmp / "props.bid", rows)
    secs, fins = [], []
    for k in range(args.warmup + args.steps):
        out = tmp / f"r{k}"
        n = int(args.ref_warmup_photons) if k < args.warmup else int(args.ref_photons)
        subprocess.run([str(exe), str(tmp / "geom.bin"), str(tmp / "props.bid"),
                        str(n), str(1796308352 + k), str(out),
                        str(exe.parent)], check=True, stdout=subprocess.DEVNULL,
                       stderr=subprocess.DEVNULL)
        raw = (tmp / f"r{k}_ref.bin").read_bytes()
        fin = int(np.frombuffer(raw, "<i8", 1)[0])
        s = float(np.frombuffer(raw, "<f8", 1, offset=8)[0])
        if k >= args.warmup:
            secs.append(s)
            fins.append(fin)
    value = sum(fins) / sum(secs)
    cores = os.cpu_count() or 1
    line = {
        "metric": "photons/s (layered tissue + vessel, 256x256x128, uniform beam, 1 B200)",
        "value": value, "unit": "photons/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(secs) / len(secs) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded layered-tissue geometry, reference input formats)",
        "config": {"workload": w.name, "photons_per_step": int(args.ref_photons),
                   "photons_per_step_note": "1e7 per step against the engine arm's 1e8, so "
                                            "that 20 steps end within minutes; the "
                                            "reference's fixed 230,400-slot drain tail "
                                            "weighs a little more at 1e7",
                   "warmup": f"{int(args.ref_warmup_photons)} photons per warm-up call",
                   "voxels": list(g.shape), "voxel_mm": g.dx, "beam": "uniform",
                   "parallelism": "single GPU (the reference has no multi-GPU path)"},
        "impl": "reference",
        "reference_run": {"value": value, "unit": "photons/s", "kind": "reference GPU binary",
                          "device": "cuda:0", "host_cores": cores,
                          "sample": f"{int(args.ref_photons)} photons per step through the "
                                    "reference's run_3dmc_gpu (its CUDA kernels on cuda:0, its "
                                    "OpenMP host tally), wall time of the call"},
        "e2e": {"value": value, "unit": "photons/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if world == 1 and not args.no_sweep:
        line["sweep"] = reference_sweep(args, exe)
    print(json.dumps(line), flush=True)


def run_batched(args):
    """One persistent launch over every job of a batched workload, timed like the
    headline (CUDA events on the launching stream, L2 flushed between steps),
    beside the same jobs launched one by one ("plain")."""
    import torch

    import ymc3d_b200 as m
    from ymc3d_b200 import workloads as W

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(dev)
    if args.workload == "homogeneous":
        w = W.homogeneous(photons=int(1e6))
    elif args.workload == "sweep":
        w = W.sweep(photon_scale=args.photon_scale, beam=args.beam)
    elif args.workload == "uneven":
        w = W.uneven(photons=max(1, int(1e7 * args.photon_scale)))
    else:
        w = W.deep_grid(photons=max(1, int(1e9 * args.photon_scale)))
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def timed(plan, steps, warmup):
        for _ in range(warmup):
            plan.execute(stream.cuda_stream)
        torch.cuda.synchronize(dev)
        ts, res = [], None
        for k in range(steps):
            flush.fill_(k & 0xff)
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.execute(stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
            res = plan.read()
        return sum(ts) / len(ts), res

    with ClockSampler(dev) as clocks:
        plan = m.Plan(w.geoms, w.props, w.jobs, math=args.math, device=dev, steps=args.step_mode,
                      use_graph=True)
        t_batch, res = timed(plan, args.steps, args.warmup)
        plan.close()
        photons = sum(r.photons for r in res)
        steps = sum(r.totals["steps"] for r in res)
        plain = None
        if len(w.jobs) > 1:
            t_plain = 0.0
            for job in w.jobs:
                pl = m.Plan([w.geoms[job.geom]], [w.props[job.props]],
                            [m.Job(0, 0, job.photons, job.seed, job.beam)], math=args.math,
                            device=dev, steps=args.step_mode)
                t, _ = timed(pl, 1, 1)
                t_plain += t
                pl.close()
            plain = {"value": photons / t_plain, "unit": "photons/s",
                     "ms_per_batch": t_plain * 1e3,
                     "how": f"{len(w.jobs)} launches, one job each, same seeds"}
    line = {"metric": f"photons/s ({w.name}, 1 B200)", "value": photons / t_batch,
            "unit": "photons/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_batch * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+u64" if args.math == "f64" else "f32+u64", "data": "synthetic (seeded)",
            "config": {"workload": w.name, "jobs": len(w.jobs), "photons_per_step": photons,
                       "math": args.math, "step_mode": args.step_mode,
                       "photon_scale": args.photon_scale,
                       "batched": "one persistent launch over all jobs, replayed from a CUDA "
                                  "graph (tally clear + kernel)"},
            "steps_per_s": steps / t_batch, "plain": plain, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def run_precision(args):
    """The precision study on the deep grid (1024x1024x256 at 0.01 mm, 256 MB, high
    albedo): the FP32 engine (fast math) against FP64 stepping, both on the same
    step mode, stated per DRS bin in sigma.  Each side is one timed launch of its
    job; the FP32 job has 1e9 * photon_scale photons and the FP64 job a quarter."""
    import torch

    import ymc3d_b200 as m
    from ymc3d_b200 import stats
    from ymc3d_b200 import workloads as W

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(dev)
    n32 = max(1, int(1e9 * args.photon_scale))
    n64 = max(1, n32 // 4)
    w = W.deep_grid(photons=n32)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    out = {}
    with ClockSampler(dev) as clocks:
        for name, math, photons, seed in (("fp32", "fast", n32, 1796308352),
                                          ("fp64", "f64", n64, 1796308353)):
            # both sides on the same step mode: the study isolates the arithmetic
            plan = m.Plan(w.geoms, w.props, [m.Job(0, 0, photons, seed, "uniform")], math=math,
                          device=dev, steps=args.step_mode)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.execute(stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            r = plan.read()[0]
            plan.close()
            out[name] = {"res": r, "s": e0.elapsed_time(e1) / 1e3}
    a, b = out["fp32"]["res"], out["fp64"]["res"]
    line = {"metric": "precision study: FP32 against FP64 stepping (deep grid, 1 B200)",
            "config": {"workload": w.name, "fp32": {"photons": n32, "math": "fast",
                                                     "step_mode": args.step_mode},
                       "fp64": {"photons": n64, "math": "f64", "step_mode": args.step_mode},
                       "photon_scale": args.photon_scale},
            "photons_per_s": {k: v["res"].photons / v["s"] for k, v in out.items()},
            "clocks": clocks.summary()}
    for f in (16, 64):
        z = stats.drs_z(a.drs, a.drs_sq, a.photons, b.drs, b.drs_sq, b.photons, f=f)
        chi2, dof, p = stats.drs_chi2(a.drs, a.drs_sq, a.photons, b.drs, b.drs_sq, b.photons, f=f)
        line[f"bins_{f}x{f}"] = {"dof": dof, "chi2": chi2, "p": p,
                                 "rms_z": float(np.sqrt(np.mean(z * z))) if z.size else None,
                                 "max_abs_z": float(np.max(np.abs(z))) if z.size else None}
    line["totals_z"] = {k: stats.total_z(a.totals, b.totals, k)
                        for k in ("r_in", "r_out", "t_in", "absorbed")}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "precision":
        run_precision(args)
    elif args.workload != "layered":
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
