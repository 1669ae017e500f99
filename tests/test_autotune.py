"""The level-schedule autotuner's output (CPU): the best row of a sweep
becomes csrc/tuned_schedule.h, and the committed header is the committed
table's best."""

import json
import os
import re

from potreeconverter_b200 import autotune


def _defines(path):
    text = open(path).read()
    return {k: int(v) for k, v in re.findall(r"#define (PCG_TUNED_\w+) (\d+)", text)}


def test_write_picks_the_fastest_schedule(tmp_path):
    rows = [
        {"schedule": [32768, 2048, 65536, 16], "ms": {"a": 10.0}, "total_ms": 10.0},
        {"schedule": [8192, 1024, 131072, 32], "ms": {"a": 9.0}, "total_ms": 9.0},
        {"schedule": [65536, 4096, 1 << 40, 8], "ms": {"a": 12.0}, "total_ms": 12.0},
        {"schedule": [16384, 1024, 65536, 8], "error": "launch failed"},
    ]
    best = autotune.write(rows, 1000, out_dir=str(tmp_path))
    assert best["schedule"] == [8192, 1024, 131072, 32]
    d = _defines(tmp_path / "tuned_schedule.h")
    assert d == {"PCG_TUNED_CTA_MIN": 8192, "PCG_TUNED_SMALL_LEVEL_CTA_MIN": 1024, "PCG_TUNED_CLUSTER_MIN": 131072,
                 "PCG_TUNED_WARP_BLOCKS_PER_SM": 32}
    table = json.load(open(tmp_path / "tuned_schedule.json"))
    assert table["points"] == 1000 and len(table["rows"]) == 4


def test_committed_header_is_the_committed_sweeps_best():
    table_path = os.path.join(autotune.CSRC, "tuned_schedule.json")
    d = _defines(os.path.join(autotune.CSRC, "tuned_schedule.h"))
    table = json.load(open(table_path))
    best = min((r for r in table["rows"] if "total_ms" in r), key=lambda r: r["total_ms"])
    assert [d["PCG_TUNED_CTA_MIN"], d["PCG_TUNED_SMALL_LEVEL_CTA_MIN"], d["PCG_TUNED_CLUSTER_MIN"],
            d["PCG_TUNED_WARP_BLOCKS_PER_SM"]] == best["schedule"]
    assert len(table["rows"]) == len(autotune.CTA_MIN) * len(autotune.SMALL_LEVEL_CTA_MIN) * len(autotune.CLUSTER_MIN) * len(
        autotune.WARP_BLOCKS)
