"""The benchmark's reference arm (CPU): `bench.py --impl reference` runs the
stock reference converter built under oracle/_ref on the benchmark's
generator and prints one JSON line in the GPU arm's terms."""

import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "PotreeConverter")),
                    reason="stock reference not built (make -C oracle ref REF=...)")
def test_reference_arm_prints_one_line_in_the_gpu_arms_terms():
    out = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--points", "100000", "--steps", "1", "--warmup", "0"],
                         cwd=REPO, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    sys.path.insert(0, REPO)
    import bench
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC and d["unit"] == "Mpts/s"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1 and d["steps"] == 1
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["points"] == 100000 and d["config"]["sampler"] == "poisson"
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
