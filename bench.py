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
         on the host cores, each step a bounded sample of the workload
  plain_form  the plain form (one launch per node, every neighbour test in
         FP64) on the same workload, one step, and the batched/plain ratio
  serving  eight jobs of 0.5-4M points submitted together to the request
         loop after one warm-up round of the same mix; p50/p99 latency from
         submit to completion, and the makespan

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
# DRAM bytes (read + write) per candidate of the acceptance kernel, from the
# ncu capture summarised in profiles/accept_hotspots-5M_poisson.md
ACCEPT_DRAM_BYTES_PER_CANDIDATE = 225.6
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


def run_reference_arm(args):
    """--impl reference: the reference's own CPU converter, all host threads."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    exe = os.path.join(REPO, "oracle", "_ref", "PotreeConverter")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference converter binary oracle/_ref/PotreeConverter not built"}))
        return
    from potreeconverter_b200 import synth
    las = synth.hotspots(REF_SAMPLE_POINTS, 1001)
    cores = os.cpu_count()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "sample.las")
        with open(path, "wb") as f:
            f.write(las)
        for w in range(args.warmup):
            cpu_reference_step(path, os.path.join(tmp, f"w{w}"))
        times = []
        for k in range(args.steps):
            pts, secs = cpu_reference_step(path, os.path.join(tmp, f"s{k}"))
            times.append(secs)
    value = REF_SAMPLE_POINTS / statistics.mean(times) / 1e6
    sample = f"{REF_SAMPLE_POINTS} points of the same generator (hotspots, seed 1001), stock reference, {cores} threads"
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": dict(WORKLOAD, sample_points=REF_SAMPLE_POINTS),
        "cpu_baseline": {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


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
    # roofline: the dominant kernel of a step (ncu launch list) is the
    # acceptance from conflict lists (greedy_list_kernel and its warp form),
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

    # ---- request loop: jobs of mixed sizes submitted together (from host
    # memory, through pcg_submit), latency = submit to completion
    serving = None
    if world == 1 and not args.no_serving:
        sizes = [500_000, 1_000_000, 2_000_000, 4_000_000] * 2
        jobs = [synth.hotspots(m, 3000 + i) for i, m in enumerate(sizes)]
        with pc.Context(device=local) as sctx:
            # warm-up: one round of the whole mix, so every worker stream,
            # its device arena and the pinned staging buffers are in use
            for j in [sctx.submit(las, method="poisson", name="warm") for las in jobs]:
                sctx.wait(j)
            t_sub, t_done, ids = {}, {}, []
            t0 = time.perf_counter()
            for i, las in enumerate(jobs):
                ids.append(sctx.submit(las, method="poisson", name=f"job{i}"))
                t_sub[i] = time.perf_counter()
            pending = set(range(len(ids)))
            while pending:
                for i in list(pending):
                    if sctx.poll(ids[i]):
                        t_done[i] = time.perf_counter()
                        pending.discard(i)
                time.sleep(0.0005)
            makespan = max(t_done.values()) - t0
            for j in ids:
                sctx.wait(j)
        lat = sorted(1e3 * (t_done[i] - t_sub[i]) for i in range(len(ids)))
        serving = {"jobs": len(sizes), "points": sizes, "sampler": "poisson", "p50_ms": statistics.median(lat),
                   "p99_ms": lat[min(len(lat) - 1, int(round(0.99 * (len(lat) - 1))))], "makespan_ms": 1e3 * makespan,
                   "mpts_per_s": sum(sizes) / (makespan * 1e6), "worker_streams": 4}

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and os.path.exists(os.path.join(REPO, "oracle", "_ref", "PotreeConverter")):
            sample = synth.hotspots(REF_SAMPLE_POINTS, 1001)
            with tempfile.TemporaryDirectory() as tmp:
                p = os.path.join(tmp, "sample.las")
                with open(p, "wb") as f:
                    f.write(sample)
                pts, secs = cpu_reference_step(p, os.path.join(tmp, "out"))
            cpu = {"value": REF_SAMPLE_POINTS / secs / 1e6, "unit": "Mpts/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"{REF_SAMPLE_POINTS} points of the same generator, stock reference converter, "
                             f"duration(chunking-total)+duration(indexing), {os.cpu_count()} threads"}
        line = {
            "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": dict(WORKLOAD, points=n, parallelism=f"replicas x{world}"),
            "e2e": {"value": e2e, "unit": "Mpts/s", "h2d_bytes_per_step": int(pinned.numel()),
                    "d2h_bytes_per_step": int(octree_bytes)},
            "gpu_launches": int(s["gpu_launches"]) * args.steps,
            "roofline": {"bound": "hbm", "kernel": "greedy_list_kernel + greedy_list_warp_kernel (all levels of a step)",
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
