"""Conversion in parts (clouds beyond the device's working set): the part
size is forced small so clouds of a few hundred thousand points run as
several parts, with the records kept on the device and streamed again from
host memory for every part, from pageable and from page-locked host
memory. Every output byte must equal the pinned reference's (golden
digests) and the one-piece form's."""

import pytest

import potreeconverter_b200 as pc
from tests.oracle_lib import las_for, load_golden, md5

pytestmark = pytest.mark.gpu

FILES = {"octree.bin": "octree", "hierarchy.bin": "hierarchy", "metadata.json": "metadata"}
NAMES = ["terrain_200k", "hotspots_300k", "duplicates_300k", "shell_400k", "centres_300k", "exact_200k", "terrain_2m",
         "lattice_2m"]
CASES = [(c, m) for c in load_golden()["cases"] if c["name"] in NAMES for m in c["outputs"]]


def _bytes(conv, f):
    v = getattr(conv, FILES[f])
    return v.encode() if isinstance(v, str) else v


@pytest.fixture(scope="module", params=["resident", "streamed"])
def parts_ctx(request):
    with pc.Context(group_points=60_000, records=request.param) as ctx:
        yield ctx


@pytest.mark.parametrize("case,method", CASES, ids=[f"{c['name']}-{m}" for c, m in CASES])
def test_parts_match_pinned_reference(parts_ctx, case, method):
    conv = parts_ctx.convert(las_for(case), method=method, name=case["name"])
    assert conv.stats["parts"] > 1 and conv.stats["survivors"] > 0
    for f in FILES:
        exp = case["outputs"][method][f]
        got = _bytes(conv, f)
        assert len(got) == exp["size"], f
        assert md5(got) == exp["md5"], f


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
@pytest.mark.parametrize("part_points", [1, 250_000, 10**9])
def test_part_sizes_match_one_piece(gpu_ctx, method, part_points):
    # one chunk per part, a few parts, and a part size above the cloud
    # (one piece): the same bytes as the one-piece conversion
    from potreeconverter_b200 import synth
    las = synth.generate("strips", 700_000, 51)
    exp = gpu_ctx.convert(las, method=method, name="s")
    with pc.Context(group_points=part_points) as ctx:
        conv = ctx.convert(las, method=method, name="s")
    assert (conv.stats["parts"] > 1) == (part_points < 700_000)
    for f in FILES:
        assert _bytes(conv, f) == _bytes(exp, f), f
    assert conv.nodes == exp.nodes


def test_parts_from_page_locked_memory(gpu_ctx):
    # the records are copied straight from page-locked host memory
    import ctypes
    import torch
    from potreeconverter_b200 import synth
    las = synth.generate("hotspots", 500_000, 52)
    host = torch.empty(len(las), dtype=torch.uint8).pin_memory()
    ctypes.memmove(host.data_ptr(), las, len(las))
    exp = gpu_ctx.convert(las, method="poisson", name="p")
    for records in ("resident", "streamed"):
        with pc.Context(group_points=100_000, records=records) as ctx:
            conv = ctx.convert((host.data_ptr(), len(las)), method="poisson", name="p")
        assert conv.stats["parts"] > 1
        for f in FILES:
            assert _bytes(conv, f) == _bytes(exp, f), (records, f)


def test_parts_write_files(tmp_path, gpu_ctx):
    # pcg_write_files joins the pieces of octree.bin
    from potreeconverter_b200 import synth
    las = synth.generate("terrain", 300_000, 53)
    with pc.Context(group_points=50_000) as ctx:
        conv = ctx.convert(las, method="poisson_average", name="w")
        ctx.write_files(las, str(tmp_path), method="poisson_average", name="w")
    assert (tmp_path / "octree.bin").read_bytes() == conv.octree
    assert (tmp_path / "hierarchy.bin").read_bytes() == conv.hierarchy
