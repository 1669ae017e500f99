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


@pytest.mark.parametrize("kind", ["terrain", "hotspots", "lattice", "strips"])
@pytest.mark.parametrize("n", [100_000, 1_000_000, 3_000_000])
def test_admission_estimate_covers_the_device_peak(gpu_ctx, kind, n):
    # the request loop admits jobs by an estimate of their device memory;
    # it must never be below what the job actually held at its peak
    las = synth.generate(kind, n, 60 + n // 100_000)
    for method in ("poisson", "poisson_average", "random"):
        st = gpu_ctx.convert_stats(las, method=method, name="fp")
        assert st["device_peak_bytes"] > 0
        assert st["device_estimate_bytes"] >= st["device_peak_bytes"], (method, st["device_peak_bytes"])


def test_large_job_ahead_of_small_jobs():
    # a large job at the head of the queue and small jobs behind it, which
    # the first-fit admission may start before it: every result is exact
    big = synth.generate("hotspots", 3_000_000, 61)
    small = [synth.generate("terrain", 100_000, 62 + i) for i in range(6)]
    with pc.Context() as ctx:
        alone = [ctx.convert(las, method="poisson", name="s").octree for las in small]
        ids = [ctx.submit(big, method="poisson", name="b")] + [ctx.submit(las, method="poisson", name="s") for las in small]
        res = [ctx.wait(j) for j in ids]
    assert [r.octree for r in res[1:]] == alone
    assert res[0].stats["num_points"] == 3_000_000
