"""Benchmark: Mpts/s of the LAS -> octree LOD build (poisson) on B200.

Workload (the configuration the headline metric is quoted on): 50M points,
LAS 1.4 point format 3 + one float32 extra attribute, 20 Gaussian hot-spots
at 100x background density over a 2 x 2 km x 50 m slab, sampler poisson,
batched form. Data is seeded synthetic (potreeconverter_b200.synth); the
reference's datasets are not available.

A step is one complete conversion of the cloud (chunking, per-chunk octree,
all sampler levels, octree.bin payloads, hierarchy.bin, metadata.json).

  value  points / device time per step with the point records resident in
         HBM and octree.bin left in HBM (CUDA events on the library's stream)
  e2e    the same conversion through the C ABI from pinned host memory, the
         host->device copy of the records and the device->host copy of
         octree.bin inside the timed region
  --impl reference   the reference converter (stock build in oracle/_ref)
         on the host cores, on the same 50M-point workload: each step one
         full conversion, at most three (minutes each on the host cores)
  plain_form  the plain form (one launch per node, every neighbour test in
         FP64) on the same workload, one step, and the batched/plain ratio
  parity   one conversion of the benchmarked cloud with each sampler, md5 of
         octree.bin, hierarchy.bin and metadata.json against the pinned
         reference's digests (tests/golden/golden.json large_cases)
  parts_form  the aerial-strip cloud (config-3 shape, poisson_average) at
         the largest size half the host memory holds (at most 3B points),
         converted in parts from page-locked host memory; Mpts/s host to
         host, beside the plain form on a 10M-point cloud of the same
         generator
  serving  the request-loop replay (config-4 shape): jobs of log-uniform
         100k-50M points (terrain generator, own seed and extent 100-2000 m,
         point format 2 or 3, samplers 60/30/10 % poisson / poisson_average
         / random) submitted at Poisson arrival times; p50/p99 latency from
         arrival to completion and the aggregate Mpts/s

Multi-GPU: the build path does not shard within one cloud (one GPU per cloud,
replicas only); with N ranks every rank converts its own seeded cloud and
value is the total points over the max-over-ranks time ("weak" scaling).
"""

from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "Mpts/s to octree (poisson)"
WORKLOAD = {"workload": "hotspots-50M", "points": 50_000_000, "las": "1.4", "point_format": 3,
            "extra_attributes": "1 x float32", "extent_m": [2000, 2000, 50], "hotspots": 20,
            "sampler": "poisson", "form": "batched", "l2": "inputs larger than L2 (1.9 GB records)"}
REF_SAMPLE_POINTS = 2_000_000
GOLDEN = os.path.join(REPO, "tests", "golden", "golden.json")
# DRAM bytes (read + write) per candidate of the acceptance kernel, from the
# ncu capture summarised in profiles/accept_hotspots-5M_poisson.md
ACCEPT_DRAM_BYTES_PER_CANDIDATE = 36.9
MEASURED_PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")


def peak_hbm():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5).stdout
                for line in out.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            for name, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_init(backend: str = "nccl"):
    """Process group for N > 1 ranks (one per GPU; gloo in the CPU tests)."""
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(minutes=10))
        return dist
    return None


def replica_seed(rank: int) -> int:
    """Each rank converts its own cloud: same generator, seed per rank."""
    return 1001 + rank


def max_over_ranks(dist, v: float, device) -> float:
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device):
    import torch
    if getattr(device, "type", "cuda") == "cuda":
        torch.cuda.synchronize(device)
    if dist is not None:
        dist.barrier()


def aggregate_mpts(world: int, points_per_rank: int, ms_per_step: float) -> float:
    """Whole-job Mpts/s: every rank's points over the max-over-ranks time."""
    return world * points_per_rank / (ms_per_step * 1e3)


def cpu_reference_step(las_path: str, outdir: str, threads: int | None = None) -> tuple[float, float]:
    """Runs the stock reference converter once; returns (points, seconds).
    Time = duration(chunking-total) + duration(indexing) from its STATS block."""
    exe = os.path.join(REPO, "oracle", "_ref", "PotreeConverter")
    env = dict(os.environ)
    t0 = time.time()
    r = subprocess.run([exe, las_path, "-o", outdir, "-m", "poisson"], capture_output=True, text=True, env=env)
    wall = time.time() - t0
    if r.returncode != 0:
        raise RuntimeError("reference converter failed: " + r.stdout[-500:] + r.stderr[-500:])
    chunk = re.search(r"duration\(chunking-total\):\s*([\d.']+)", r.stdout)
    index = re.search(r"duration\(indexing\):\s*([\d.']+)", r.stdout)
    pts = re.search(r"#points:\s*([\d']+)", r.stdout)
    secs = (float(chunk.group(1).replace("'", "")) + float(index.group(1).replace("'", ""))) if chunk and index else wall
    return float(pts.group(1).replace("'", "")) if pts else float("nan"), secs


REF_TIME_BUDGET_S = 420.0


def run_reference_arm(args):
    """--impl reference: the reference's own CPU converter (stock build), all
    host threads, on the benchmarked workload itself (the 50M-point hot-spot
    cloud, seed 1001). One conversion takes minutes on the host cores, so a
    step is one full conversion and the run times at most min(steps, 3) of
    them, stopping early when the next one would pass REF_TIME_BUDGET_S;
    value is the median. The warm-up is the write of the file (page cache)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    exe = os.path.join(REPO, "oracle", "_ref", "PotreeConverter")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference converter binary oracle/_ref/PotreeConverter not built"}))
        return
    from potreeconverter_b200 import synth
    n = args.points
    las = synth.hotspots(n, replica_seed(0))
    cores = os.cpu_count()
    times = []
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cloud.las")
        with open(path, "wb") as f:
            f.write(las)
        del las
        t0 = time.perf_counter()
        for k in range(max(1, min(args.steps, 3))):
            if times and (time.perf_counter() - t0) + max(times) > REF_TIME_BUDGET_S:
                break
            pts, secs = cpu_reference_step(path, os.path.join(tmp, f"s{k}"))
            times.append(secs)
            subprocess.run(["rm", "-rf", os.path.join(tmp, f"s{k}")], check=False)
    secs = statistics.median(times)
    value = n / secs / 1e6
    sample = (f"the whole workload ({n} points, hotspots seed 1001), stock reference, duration(chunking-total)+"
              f"duration(indexing), median of {len(times)} full conversions, {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": args.gpus, "steps": len(times),
        "steps_requested": args.steps, "warmup": 0, "ms_per_step": 1e3 * secs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(WORKLOAD, points=n),
        "cpu_baseline": {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def parity_leg(ctx, pinned, n):
    """md5 of the three outputs of the benchmarked cloud with each sampler
    against the pinned reference's digests (golden large_cases)."""
    import hashlib
    try:
        with open(GOLDEN) as f:
            case = next(c for c in json.load(f).get("large_cases", []) if c["name"] == "hotspots_50m")
    except (OSError, StopIteration):
        return {"md5_match": None, "why": "no golden digests for the 50M hot-spot cloud"}
    if n != case["points"]:
        return {"md5_match": None, "why": f"workload of {n} points, digests for {case['points']}"}
    las_md5 = hashlib.md5(memoryview(pinned.numpy())).hexdigest()
    out = {"las_md5_match": las_md5 == case["las_md5"], "samplers": {}}
    for method in ("poisson", "poisson_average", "random"):
        conv = ctx.convert((pinned.data_ptr(), pinned.numel()), method=method, name=case["name"])
        got = {"octree.bin": conv.octree, "hierarchy.bin": conv.hierarchy, "metadata.json": conv.metadata.encode()}
        out["samplers"][method] = all(hashlib.md5(got[f]).hexdigest() == case["outputs"][method][f]["md5"] for f in got)
        del conv, got
    out["md5_match"] = out["las_md5_match"] and all(out["samplers"].values())
    out["reference"] = "pinned reference digests, tests/golden/golden.json large_cases hotspots_50m"
    return out


def host_points_budget(bytes_per_point: float) -> int:
    """Points whose page-locked input and output fit half the host memory
    available now."""
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) * 1024 for l in f if l.startswith("MemAvailable"))
    except (OSError, StopIteration):
        avail = 64 << 30
    return int(avail / 2 / bytes_per_point)


def parts_leg(local, stream, points, steps):
    """Config-3 shape: the aerial-strip cloud, poisson_average, converted in
    parts from page-locked host memory; Mpts/s from host records to the
    three outputs in host memory (the pieces of octree.bin included)."""
    import torch
    import potreeconverter_b200 as pc
    from potreeconverter_b200 import synth_gpu
    t0 = time.perf_counter()
    img = synth_gpu.strips(points, 1003, device=torch.device("cuda", local))
    gen_s = time.perf_counter() - t0
    out = {"workload": "strips", "points": points, "point_format": 3, "sampler": "poisson_average",
           "extent_m": [20000, 20000], "strips": 40, "generator": "potreeconverter_b200.synth_gpu.strips seed 1003",
           "generate_s": round(gen_s, 1)}
    try:
        with pc.Context(device=local, stream=stream.cuda_stream) as ctx:
            st = ctx.convert_stats((img.data_ptr(), img.numel()), method="poisson_average", name="strips")  # warm-up
            times = []
            for _ in range(steps):
                t = time.perf_counter()
                st = ctx.convert_stats((img.data_ptr(), img.numel()), method="poisson_average", name="strips")
                times.append(time.perf_counter() - t)
    except Exception as e:  # the leg reports what it reached
        out["error"] = f"{type(e).__name__}: {e}"
        return out
    ms = 1e3 * statistics.median(times)
    out.update({"value": points / (ms * 1e3), "unit": "Mpts/s", "ms_per_step": ms, "steps": steps,
                "parts": int(st["parts"]), "survivors": int(st["survivors"]), "records_resident": bool(st["records_resident"]),
                "device_peak_gb": round(st["device_peak_bytes"] / 1e9, 2), "output_points": int(st["output_points"]),
                "h2d_bytes_per_step": int(img.numel()), "d2h_bytes_per_step": int(st["octree_size"]),
                "stages_ms": {k: round(st[k], 1) for k in ("ms_h2d", "ms_chunking", "ms_octree", "ms_sampling", "ms_output",
                                                          "ms_d2h", "ms_host_writers", "ms_total")}})
    del img
    # the plain form on a cloud of the same generator (one launch per node,
    # every neighbour test in FP64), 10M points
    pn = 10_000_000
    small = synth_gpu.strips(pn, 1003, device=torch.device("cuda", local))
    with pc.Context(device=local, stream=stream.cuda_stream, form="plain") as pctx:
        t = time.perf_counter()
        pctx.convert_stats((small.data_ptr(), small.numel()), method="poisson_average", name="strips")
        p_s = time.perf_counter() - t
    with pc.Context(device=local, stream=stream.cuda_stream) as bctx:
        bctx.convert_stats((small.data_ptr(), small.numel()), method="poisson_average", name="strips")
        t = time.perf_counter()
        bctx.convert_stats((small.data_ptr(), small.numel()), method="poisson_average", name="strips")
        b_s = time.perf_counter() - t
    out["plain_form_10M"] = {"value": pn / (p_s * 1e6), "unit": "Mpts/s", "batched_value": pn / (b_s * 1e6),
                             "batched_over_plain": p_s / b_s}
    out["parts_over_plain"] = out["value"] / (pn / (p_s * 1e6))
    return out


def serving_leg(local, jobs: int, rate: float, seed: int = 2000):
    """Config-4 shape replay: `jobs` jobs with Poisson arrivals at `rate`
    jobs/s (log-uniform 100k-50M points, terrain generator with its own seed
    and extent 100-2000 m, point format 2 or 3, samplers 60/30/10 %),
    submitted at their arrival times; latency = arrival to completion."""
    import numpy as np
    import torch
    import potreeconverter_b200 as pc
    from potreeconverter_b200 import synth_gpu
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(1e5), np.log(5e7), jobs)).astype(np.int64)
    extents = rng.uniform(100.0, 2000.0, jobs)
    methods = rng.choice(["poisson", "poisson_average", "random"], jobs, p=[0.6, 0.3, 0.1])
    pdrfs = rng.choice([2, 3], jobs)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, jobs))
    dev = torch.device("cuda", local)
    t0 = time.perf_counter()
    images = [synth_gpu.terrain(int(sizes[j]), seed + j, float(extents[j]), int(pdrfs[j]), device=dev) for j in range(jobs)]
    gen_s = time.perf_counter() - t0
    with pc.Context(device=local) as ctx:
        # warm-up: the worker streams, their arenas and the pinned pool
        for j in [ctx.submit((images[i].data_ptr(), images[i].numel()), method=methods[i], name="w") for i in range(min(8, jobs))]:
            ctx.wait(j)
        ids, t_done = [None] * jobs, [None] * jobs
        start = time.perf_counter()
        nxt = 0
        pending = set()
        while nxt < jobs or pending:
            now = time.perf_counter() - start
            while nxt < jobs and arrivals[nxt] <= now:
                ids[nxt] = ctx.submit((images[nxt].data_ptr(), images[nxt].numel()), method=methods[nxt], name=f"job{nxt}")
                pending.add(nxt)
                nxt += 1
            for i in list(pending):
                if ctx.poll(ids[i]):
                    t_done[i] = time.perf_counter() - start
                    pending.discard(i)
            time.sleep(0.0005)
        makespan = max(t_done)
        for j in ids:
            ctx.wait(j)
    del images
    lat = np.array([1e3 * (t_done[i] - arrivals[i]) for i in range(jobs)])
    return {"jobs": jobs, "arrival_rate_per_s": rate, "offered_mpts_per_s": float(sizes.sum() / arrivals[-1] / 1e6),
            "points_total": int(sizes.sum()), "sizes": "log-uniform 100k-50M", "samplers": "60/30/10 % poisson/poisson_average/random",
            "point_formats": [2, 3], "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_ms": float(lat.max()), "makespan_s": makespan, "mpts_per_s": float(sizes.sum() / makespan / 1e6),
            "worker_streams": 4, "generate_s": round(gen_s, 1),
            "time_compression": f"{rate / 4.0:g}x the configuration's 4 jobs/s, {jobs} of its 2,000 jobs"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--points", type=int, default=WORKLOAD["points"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-form leg (one-launch-per-node form)")
    ap.add_argument("--no-serving", action="store_true", help="skip the request-loop latency leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the md5 check against the pinned reference")
    ap.add_argument("--no-parts", action="store_true", help="skip the conversion-in-parts leg (config-3 shape)")
    ap.add_argument("--parts-points", type=int, default=0, help="points of the parts leg (0: as many as host memory holds, <= 3B)")
    ap.add_argument("--serving-jobs", type=int, default=200)
    ap.add_argument("--serving-rate", type=float, default=4.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args)
        return

    import numpy as np
    import torch

    import potreeconverter_b200 as pc
    from potreeconverter_b200 import synth

    dist = dist_init()
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    n = args.points
    las = synth.hotspots(n, replica_seed(rank))
    off = int.from_bytes(las[96:100], "little")
    header = las[:off]
    pinned = torch.empty(len(las), dtype=torch.uint8, pin_memory=True)
    pinned.numpy()[:] = np.frombuffer(las, dtype=np.uint8)
    records = torch.from_numpy(np.frombuffer(las, dtype=np.uint8, offset=off).copy()).to(device)
    del las

    stream = torch.cuda.Stream(device=device)
    ctx = pc.Context(device=local, stream=stream.cuda_stream)

    # ---- value: records resident in HBM, octree.bin left in HBM
    for _ in range(args.warmup):
        ctx.convert_resident(header, records.data_ptr(), method="poisson", name="bench")
    barrier(dist, device)
    stats = []
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            stats.append(ctx.convert_resident(header, records.data_ptr(), method="poisson", name="bench"))
        end.record(stream)
        end.synchronize()
    barrier(dist, device)
    ms = start.elapsed_time(end) / args.steps
    ms = max_over_ranks(dist, ms, device)
    value = aggregate_mpts(world, n, ms)

    # ---- e2e: through the C ABI from pinned host memory
    for _ in range(max(1, args.warmup // 2)):
        ctx.convert_stats((pinned.data_ptr(), pinned.numel()), method="poisson", name="bench")
    barrier(dist, device)
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    octree_bytes = 0
    e_stats = None
    e_start.record(stream)
    for _ in range(args.steps):
        e_stats = ctx.convert_stats((pinned.data_ptr(), pinned.numel()), method="poisson", name="bench")
        octree_bytes = e_stats["octree_size"]
    e_end.record(stream)
    e_end.synchronize()
    barrier(dist, device)
    e_ms = max_over_ranks(dist, e_start.elapsed_time(e_end) / args.steps, device)
    e2e = aggregate_mpts(world, n, e_ms)

    s = stats[-1]
    rec_len = int.from_bytes(header[105:107], "little")
    bpp = 39
    out_pts = s["output_points"]
    # roofline: the largest kernel family of a step (ncu launch list, 25 %)
    # is the acceptance from conflict lists (greedy_list_cluster_kernel for
    # the largest nodes, greedy_list_kernel, greedy_list_warp_kernel),
    # launched once per octree level. Algorithmic bytes: per candidate its
    # record (16 B), list length (1 B) and its decision, rank and flag
    # (9 B); per list entry the entry (4 B) and that candidate's decision
    # (4 B). Duration: the acceptance device time of the step (ms_greedy
    # minus the list builds), all levels.
    accept_ms = s["ms_greedy"] - s["ms_lists"]
    accept_bytes = s["candidates"] * 26 + s["list_entries"] * 8
    peak, peak_kind = peak_hbm()
    achieved = accept_bytes / (accept_ms * 1e-3) / 1e9 if accept_ms > 0 else 0.0
    traffic = s["candidates"] * ACCEPT_DRAM_BYTES_PER_CANDIDATE if ACCEPT_DRAM_BYTES_PER_CANDIDATE else None
    whole_bytes = n * rec_len + out_pts * bpp  # B_alg: read every record once, write every output record once
    # ---- plain form on the same workload (one step, single GPU runs only):
    # one launch per node, every neighbour test in FP64; the batched form
    # above is measured against it
    plain = None
    if world == 1 and not args.no_plain:
        pctx = pc.Context(device=local, stream=stream.cuda_stream, form="plain")
        p_start = torch.cuda.Event(enable_timing=True)
        p_end = torch.cuda.Event(enable_timing=True)
        p_start.record(stream)
        pctx.convert_resident(header, records.data_ptr(), method="poisson", name="bench")
        p_end.record(stream)
        p_end.synchronize()
        p_ms = p_start.elapsed_time(p_end)
        pctx.close()
        plain = {"value": n / (p_ms * 1e3), "unit": "Mpts/s", "ms_per_step": p_ms, "steps": 1,
                 "batched_over_plain": (n / (ms * 1e3)) / (n / (p_ms * 1e3))}

    # ---- parity of the benchmarked workload (one conversion per sampler,
    # outside the timed region)
    def leg(fn, *a):
        # a failing side leg is reported in the line, not fatal to it
        try:
            return fn(*a)
        except Exception as e:  # noqa: BLE001
            return {"error": f"{type(e).__name__}: {e}"}

    parity = None
    if rank == 0 and not args.no_parity:
        parity = leg(parity_leg, ctx, pinned, n)

    # ---- the request-loop replay (config-4 shape) and the conversion in
    # parts (config-3 shape), single GPU runs only
    serving = None
    if world == 1 and not args.no_serving:
        serving = leg(serving_leg, local, args.serving_jobs, args.serving_rate)
    parts = None
    if world == 1 and not args.no_parts:
        # page-locked input (34 B) and octree.bin pieces (about 1.9 output
        # points of 34 B per input point) in half the available host memory
        pts = args.parts_points or min(3_000_000_000, host_points_budget(34 + 34 * 1.9))
        parts = leg(parts_leg, local, stream, pts, 1)

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and os.path.exists(os.path.join(REPO, "oracle", "_ref", "PotreeConverter")):
            sample = synth.hotspots(REF_SAMPLE_POINTS, 1001)
            with tempfile.TemporaryDirectory() as tmp:
                p = os.path.join(tmp, "sample.las")
                with open(p, "wb") as f:
                    f.write(sample)
                secs = statistics.median(cpu_reference_step(p, os.path.join(tmp, f"out{k}"))[1] for k in range(3))
            cpu = {"value": REF_SAMPLE_POINTS / secs / 1e6, "unit": "Mpts/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"{REF_SAMPLE_POINTS} points of the same generator, stock reference converter, "
                             f"duration(chunking-total)+duration(indexing), median of 3, {os.cpu_count()} threads"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(WORKLOAD, points=n, parallelism=f"replicas x{world}"),
            "e2e": {"value": e2e, "unit": "Mpts/s", "h2d_bytes_per_step": int(pinned.numel()),
                    "d2h_bytes_per_step": int(octree_bytes)},
            "gpu_launches": int(s["gpu_launches"]) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "greedy_list_cluster_kernel + greedy_list_kernel + greedy_list_warp_kernel (list acceptance, all levels of a step)",
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "traffic_source": "DRAM bytes per candidate from ncu, profiles/accept_hotspots-5M_poisson.md",
                         "algorithmic_bytes": accept_bytes, "kernel_ms": accept_ms,
                         "pipeline_achieved": whole_bytes / (ms * 1e-3) / 1e9, "pipeline_bytes_per_step": whole_bytes},
            "stages_ms": {k: round(s[k], 3) for k in ("ms_chunking", "ms_octree", "ms_sampling", "ms_sort", "ms_greedy", "ms_lists",
                                                     "ms_output", "ms_host_writers")},
            "e2e_stages_ms": {k: round(e_stats[k], 3) for k in ("ms_total", "ms_h2d", "ms_sampling", "ms_output", "ms_d2h",
                                                                  "ms_host_writers")},
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "plain_form": plain,
            "parity": parity,
            "parts_form": parts,
            "serving": serving,
            "escalated_pairs": int(s["escalated_pairs"]),
            "sampler": {k: int(s[k]) for k in ("sampled_nodes", "candidates", "replayed_nodes", "replayed_candidates",
                                               "heapsort_fallbacks", "list_entries")},
        }
        print(json.dumps(line))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
