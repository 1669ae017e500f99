"""Full-size parity against the pinned reference (golden `large_cases`,
made by tests/golden/make_golden.py --large-only):

* the hot-spot cloud of the benchmark at 10M points (all three samplers, one
  piece) and at its full 50M points (all three samplers, in parts of at
  most 20M points with resident records);
* the 100M-point precision-stress lattice (poisson): every acceptance and
  output byte equal to the reference's, with the count of pairs the FP32
  prefilter left to FP64 reported;
* a 20M-point aerial-strip cloud, in one piece and in parts whose records
  are streamed from host memory again for every part.

md5 equality of octree.bin and hierarchy.bin means every node holds the
reference's points in the reference's order: zero acceptance mismatches."""

import functools
import hashlib

import pytest

import potreeconverter_b200 as pc
from tests.oracle_lib import load_golden

pytestmark = pytest.mark.gpu

LARGE = {c["name"]: c for c in load_golden().get("large_cases", [])}
FILES = {"octree.bin": "octree", "hierarchy.bin": "hierarchy", "metadata.json": "metadata"}


@functools.lru_cache(maxsize=2)
def _las_named(name):
    from potreeconverter_b200 import synth
    case = LARGE[name]
    las = synth.generate(case["kind"], case["points"], case["seed"], **case["kwargs"])
    assert hashlib.md5(las).hexdigest() == case["las_md5"], "synthetic generator output changed"
    return las


def _las(case):
    return _las_named(case["name"])


def _check(conv, case, method):
    differ = []
    for f, attr in FILES.items():
        v = getattr(conv, attr)
        v = v.encode() if isinstance(v, str) else v
        exp = case["outputs"][method][f]
        if len(v) != exp["size"] or hashlib.md5(v).hexdigest() != exp["md5"]:
            differ.append(f)
    assert not differ, f"{case['name']} {method}: {differ} differ from the pinned reference"


def _need(name):
    if name not in LARGE:
        pytest.skip(f"golden large case {name} not generated")
    return LARGE[name]


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_hotspots_10m_matches_reference(gpu_ctx, method):
    case = _need("hotspots_10m")
    _check(gpu_ctx.convert(_las(case), method=method, name=case["name"]), case, method)


def test_hotspots_50m_random_matches_reference(gpu_ctx):
    """Above 5M chunk-root points under a parent the chunk roots are tasks of
    their own and the random sampler shuffles each of them a second time."""
    case = _need("hotspots_50m")
    _check(gpu_ctx.convert(_las(case), method="random", name=case["name"]), case, "random")


def test_hotspots_50m_in_parts_matches_reference():
    case = _need("hotspots_50m")
    las = _las(case)
    with pc.Context(group_points=20_000_000, records="resident") as ctx:
        for method in ("poisson", "poisson_average", "random"):
            conv = ctx.convert(las, method=method, name=case["name"])
            assert conv.stats["parts"] >= 3
            _check(conv, case, method)


def test_lattice_100m_precision_stress_matches_reference(gpu_ctx):
    case = _need("lattice_100m")
    conv = gpu_ctx.convert(_las(case), method="poisson", name=case["name"])
    _check(conv, case, "poisson")
    print(f"lattice 100M: {conv.stats['escalated_pairs']} pairs decided in FP64 after the FP32 prefilter, "
          f"{conv.stats['candidates']} candidates, 0 acceptance mismatches")
    assert conv.stats["escalated_pairs"] > 0


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_strips_20m_matches_reference(gpu_ctx, method):
    case = _need("strips_20m")
    las = _las(case)
    _check(gpu_ctx.convert(las, method=method, name=case["name"]), case, method)
    with pc.Context(group_points=4_000_000, records="streamed") as ctx:
        conv = ctx.convert(las, method=method, name=case["name"])
    assert conv.stats["parts"] >= 4 and conv.stats["records_resident"] == 0
    _check(conv, case, method)
