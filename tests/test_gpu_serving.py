"""Request loop (pcg_submit / pcg_poll / pcg_wait): jobs of different sizes
and samplers submitted together run side by side on the worker streams, and
every result is byte-identical to the same job converted alone."""

import pytest

import potreeconverter_b200 as pc
from potreeconverter_b200 import synth

pytestmark = pytest.mark.gpu

MIX = [("terrain", 300_000, 51, "poisson"), ("hotspots", 800_000, 52, "poisson"), ("cube", 200_000, 53, "poisson_average"),
       ("lattice", 400_000, 54, "random"), ("strips", 150_000, 55, "poisson"), ("terrain", 50_000, 56, "poisson_average")]


def _files(conv):
    return conv.octree, conv.hierarchy, conv.metadata


def test_each_result_in_the_mix_equals_the_result_alone(gpu_ctx):
    inputs = [(synth.generate(kind, n, seed), method) for kind, n, seed, method in MIX]
    alone = [_files(gpu_ctx.convert(las, method=m, name=f"job{i}")) for i, (las, m) in enumerate(inputs)]
    with pc.Context() as ctx:
        ids = [ctx.submit(las, method=m, name=f"job{i}") for i, (las, m) in enumerate(inputs)]
        mixed = [_files(ctx.wait(j)) for j in ids]
    for i, (a, b) in enumerate(zip(alone, mixed)):
        assert a == b, f"job {i} ({MIX[i]}) differs in the mix"


def test_poll_reports_completion_and_unknown_jobs_fail(gpu_ctx):
    las = synth.generate("terrain", 20_000, 57)
    with pc.Context() as ctx:
        j = ctx.submit(las, method="poisson", name="one")
        conv = ctx.wait(j)
        assert conv.octree
        with pytest.raises(pc.PcgError):
            ctx.poll(j + 1000)
