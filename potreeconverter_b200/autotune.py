"""Autotuner of the samplers' level schedule (csrc/sampling.h LevelSchedule):
which nodes of a level get a CTA, a cluster of CTAs or a warp, and how many
resident blocks per SM pull warp-sized nodes from the device work queue.

Run on the target GPU:

    python -m potreeconverter_b200.autotune [--points N] [--write]

Each candidate schedule is set through the PCG_SCHEDULE override (the
library reads it at every level) and times the benchmark's hot-spot cloud
and a terrain cloud with the poisson and poisson_average samplers, records
device-resident: the median device time of three conversions after one
warm-up. The schedule with the smallest
summed time wins; --write stores it in csrc/tuned_schedule.h (rebuild the
library afterwards) and the whole table in csrc/tuned_schedule.json.
"""

from __future__ import annotations

import argparse
import itertools
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")

CTA_MIN = [8192, 16384, 32768, 65536]
SMALL_LEVEL_CTA_MIN = [1024, 2048, 4096]
CLUSTER_MIN = [65536, 131072, 1 << 40]
WARP_BLOCKS = [8, 16, 32]


def sweep(points: int) -> list:
    import statistics
    import numpy as np
    import torch
    import potreeconverter_b200 as pc
    from potreeconverter_b200 import synth
    stream = torch.cuda.Stream()
    clouds = []
    for kind, n, seed in (("hotspots", points, 1001), ("terrain", points // 2, 1000)):
        las = synth.generate(kind, n, seed)
        off = int.from_bytes(las[96:100], "little")
        recs = torch.from_numpy(np.frombuffer(las, dtype=np.uint8, offset=off).copy()).cuda()
        clouds.append((kind, las[:off], recs))
    rows = []
    with pc.Context(stream=stream.cuda_stream) as ctx:
        for cta, small, clu, warp in itertools.product(CTA_MIN, SMALL_LEVEL_CTA_MIN, CLUSTER_MIN, WARP_BLOCKS):
            os.environ["PCG_SCHEDULE"] = f"{cta},{small},{clu},{warp}"
            ms = {}
            for kind, header, recs in clouds:
                for method in ("poisson", "poisson_average"):
                    ctx.convert_resident(header, recs.data_ptr(), method=method, name="t")
                    times = []
                    for _ in range(3):
                        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                        a.record(stream)
                        ctx.convert_resident(header, recs.data_ptr(), method=method, name="t")
                        b.record(stream)
                        b.synchronize()
                        times.append(a.elapsed_time(b))
                    ms[f"{kind}-{method}"] = statistics.median(times)
            rows.append({"schedule": [cta, small, clu, warp], "ms": ms, "total_ms": sum(ms.values())})
            print(json.dumps(rows[-1]), flush=True)
    os.environ.pop("PCG_SCHEDULE", None)
    return rows


def write(rows: list, points: int, out_dir: str = CSRC):
    ok = [r for r in rows if "total_ms" in r]
    best = min(ok, key=lambda r: r["total_ms"])
    cta, small, clu, warp = best["schedule"]
    with open(os.path.join(out_dir, "tuned_schedule.h"), "w") as f:
        f.write("// Level schedule of the samplers (sampling.h LevelSchedule). Written by\n"
                "// potreeconverter_b200/autotune.py from a sweep on the target GPU; the\n"
                "// values below are the sweep's best for the benchmarked workload, or the\n"
                "// hand-set defaults until a sweep has run.\n#pragma once\n"
                f"#define PCG_TUNED_CTA_MIN {cta}\n#define PCG_TUNED_SMALL_LEVEL_CTA_MIN {small}\n"
                f"#define PCG_TUNED_CLUSTER_MIN {clu}\n#define PCG_TUNED_WARP_BLOCKS_PER_SM {warp}\n")
    with open(os.path.join(out_dir, "tuned_schedule.json"), "w") as f:
        json.dump({"points": points, "best": best, "rows": rows}, f, indent=1)
    return best


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--points", type=int, default=20_000_000)
    ap.add_argument("--write", action="store_true")
    args = ap.parse_args()
    rows = sweep(args.points)
    if args.write:
        print(json.dumps({"best": write(rows, args.points)}))


if __name__ == "__main__":
    main()
