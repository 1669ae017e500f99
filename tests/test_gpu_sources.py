"""Several input files and --attributes lists through the C ABI: the CUDA
pipeline's octree.bin, hierarchy.bin and metadata.json are byte-identical to
the pinned reference's (golden digests of multi-source cases) and to the
oracle on fresh inputs: tiles in point formats 0-3 with their own scales,
offsets and extra bytes, in any order, filtered to any attribute list whose
result the reference defines. Lists it leaves undefined are refused."""

import os
import subprocess

import numpy as np
import pytest

import potreeconverter_b200 as pc
from tests.oracle_lib import load_golden, md5, sources_for

pytestmark = pytest.mark.gpu

MULTI = [(c, m) for c in load_golden()["multi_cases"] for m in c["outputs"]]
FILES = {"octree.bin": "octree", "hierarchy.bin": "hierarchy", "metadata.json": "metadata"}
STANDARD = ["intensity", "return number", "number of returns", "classification", "scan angle rank", "user data",
            "point source id", "gps-time", "rgb"]


def _bytes(conv, f):
    v = getattr(conv, FILES[f])
    return v.encode() if isinstance(v, str) else v


def _same(conv, exp):
    for f in FILES:
        assert _bytes(conv, f) == exp[f], f


@pytest.mark.parametrize("case,method", MULTI, ids=[f"{c['name']}-{m}" for c, m in MULTI])
def test_sources_match_pinned_reference(gpu_ctx, case, method):
    conv = gpu_ctx.convert(sources_for(case), method=method, name=case["meta_name"], attributes=case["attributes"])
    for f in FILES:
        got = _bytes(conv, f)
        exp = case["outputs"][method][f]
        assert len(got) == exp["size"], f
        assert md5(got) == exp["md5"], f


@pytest.mark.parametrize("case,method", [(c, m) for c, m in MULTI if c["points"] <= 300_000],
                         ids=[f"{c['name']}-{m}" for c, m in MULTI if c["points"] <= 300_000])
def test_plain_form_sources_match_pinned_reference(case, method):
    with pc.Context(form="plain") as ctx:
        conv = ctx.convert(sources_for(case), method=method, name=case["meta_name"], attributes=case["attributes"])
    for f in FILES:
        assert md5(_bytes(conv, f)) == case["outputs"][method][f]["md5"], f


@pytest.mark.parametrize("seed", [101, 102, 103])
@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_fresh_tiles_match_oracle(gpu_ctx, oracle, seed, method):
    from potreeconverter_b200 import synth
    rng = np.random.default_rng(seed)
    tiles = synth.tiles(300_000, seed)
    order = [int(k) for k in rng.permutation(len(tiles))][: int(rng.integers(2, len(tiles) + 1))]
    srcs = [tiles[k] for k in order]
    exp = oracle.convert_sources(srcs, method, name="fresh")
    _same(gpu_ctx.convert(srcs, method=method, name="fresh"), exp)


@pytest.mark.parametrize("seed", [201, 202, 203, 204])
@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_fresh_attribute_lists_match_oracle(gpu_ctx, oracle, seed, method):
    # seeded subsets of the standard attributes in seeded order (rgb kept for
    # poisson_average, which averages it), over tiles whose extra bytes are
    # then not kept
    from potreeconverter_b200 import synth
    rng = np.random.default_rng(seed)
    names = [STANDARD[int(k)] for k in rng.permutation(len(STANDARD))][: int(rng.integers(1, len(STANDARD) + 1))]
    if method == "poisson_average" and "rgb" not in names:
        names.append("rgb")
    srcs = synth.tiles(200_000, seed)
    exp = oracle.convert_sources(srcs, method, name="attrs", attributes=names)
    _same(gpu_ctx.convert(srcs, method=method, name="attrs", attributes=names), exp)


def test_one_source_given_as_a_list_equals_the_plain_job(gpu_ctx):
    from potreeconverter_b200 import synth
    las = synth.hotspots(150_000, 7)
    a = gpu_ctx.convert(las, method="poisson", name="h")
    b = gpu_ctx.convert([las], method="poisson", name="h")
    for f in FILES:
        assert _bytes(a, f) == _bytes(b, f), f


def test_empty_source_among_others(gpu_ctx, oracle):
    # a file without points adds its attributes and header box; rgb, which
    # only it has, gets the reference's statistics of no values (+inf)
    from potreeconverter_b200 import synth
    srcs = synth.sources("tiles_empty", 100_000, 9)
    for method in ("poisson", "random"):
        exp = oracle.convert_sources(srcs, method, name="e")
        assert b"[inf, inf, inf]" in exp["metadata.json"]
        _same(gpu_ctx.convert(srcs, method=method, name="e"), exp)


def test_undefined_attribute_lists_are_refused(gpu_ctx):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(20_000, 3)
    cases = [
        (tiles, "poisson", ["amplitude"]),              # extra written past the point record
        (tiles[:2], "poisson_average", ["intensity"]),  # no rgb to average
        (tiles[:2], "poisson", ["rgb", "rgb"]),         # listed twice
        (tiles[:2], "poisson", ["position"]),           # position is always first
    ]
    for srcs, method, names in cases:
        with pytest.raises(pc.PcgError) as e:
            gpu_ctx.convert(srcs, method=method, attributes=names)
        assert e.value.status == 1, names


def test_bad_source_is_named(gpu_ctx):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(20_000, 3)
    with pytest.raises(pc.PcgError) as e:
        gpu_ctx.convert([tiles[0], b"not a las file" * 30], method="poisson")
    assert e.value.status == 1 and "source 1" in str(e.value)


def test_request_loop_takes_sources_and_attributes(gpu_ctx):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(200_000, 21)
    names = ["rgb", "classification"]
    ids = [gpu_ctx.submit(tiles, method="poisson_average", name="q", attributes=names),
           gpu_ctx.submit(tiles[0], method="poisson", name="q")]
    alone = [gpu_ctx.convert(tiles, method="poisson_average", name="q", attributes=names),
             gpu_ctx.convert(tiles[0], method="poisson", name="q")]
    for jid, exp in zip(ids, alone):
        got = gpu_ctx.wait(jid)
        for f in FILES:
            assert _bytes(got, f) == _bytes(exp, f), f


def test_cli_converts_a_directory_of_tiles(tmp_path, oracle):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(200_000, 31)
    d = tmp_path / "tiles"
    d.mkdir()
    for k, img in enumerate(tiles):
        (d / f"t{k}.las").write_bytes(img)
    (d / "notes.txt").write_text("not an input")
    out = tmp_path / "out"
    exe = os.path.join(os.path.dirname(pc.__file__), "PotreeConverter")
    r = subprocess.run([exe, str(d), "-o", str(out), "-m", "poisson", "--attributes", "rgb", "gps-time", "intensity"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    exp = oracle.convert_sources(tiles, "poisson", name="tiles", attributes=["rgb", "gps-time", "intensity"])
    for f in FILES:
        assert (out / f).read_bytes() == exp[f], f


def test_sources_with_records_on_the_device(gpu_ctx):
    # pcg_source.device_records: headers on the host, decoded records already
    # in device memory (a LAZ header too), mixed with host images
    import struct
    import torch
    from potreeconverter_b200 import synth
    from tests.oracle_lib import have_laz_tool, to_laz
    tiles = synth.tiles(200_000, 51)
    exp = gpu_ctx.convert(tiles, method="poisson", name="d")
    keep, srcs = [], []
    for k, img in enumerate(tiles):
        if k == 1:
            srcs.append(img)  # a host image among them
            continue
        off = struct.unpack_from("<I", img, 96)[0]
        rec = torch.frombuffer(bytearray(img[off:]), dtype=torch.uint8).cuda()
        keep.append(rec)
        header = img[:off]
        if k == 2 and have_laz_tool():
            laz = to_laz(img)
            header = laz[:struct.unpack_from("<I", laz, 96)[0]]
        srcs.append(pc.Resident(header, rec.data_ptr()))
    torch.cuda.synchronize()
    got = gpu_ctx.convert(srcs, method="poisson", name="d")
    for f in FILES:
        assert _bytes(got, f) == _bytes(exp, f), f
