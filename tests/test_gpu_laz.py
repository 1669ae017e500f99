"""LAZ inputs on the device: the decode kernel reproduces LASzip's point
records byte for byte, and conversions of .laz sources match the pinned
reference's digests for the same .laz files (golden multi-source cases with
a "laz" entry) and the conversion of the LAS files they were made from.
LAZ files come from the reference's vendored LASzip (oracle/_ref/laz_tool)."""

import os
import subprocess
import time

import numpy as np
import pytest

import potreeconverter_b200 as pc
from tests.oracle_lib import have_laz_tool, las_records, laz_sources_for, load_golden, md5, to_laz

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_laz_tool(), reason="oracle/_ref/laz_tool not built (make -C oracle ref REF=<reference tree>)")]

LAZ_CASES = [(c, m) for c in load_golden()["multi_cases"] if c.get("laz") for m in c["outputs"]]
FILES = {"octree.bin": "octree", "hierarchy.bin": "hierarchy", "metadata.json": "metadata"}


def _bytes(conv, f):
    v = getattr(conv, FILES[f])
    return v.encode() if isinstance(v, str) else v


@pytest.mark.parametrize("chunk_size", [0, 1000, 7777])
def test_device_decode_matches_laszip(gpu_ctx, chunk_size):
    from potreeconverter_b200 import synth
    inputs = [(f"tile{k}", t) for k, t in enumerate(synth.tiles(240_000, 78))]
    inputs += [("hotspots", synth.generate("hotspots", 150_000, 6)), ("strips", synth.generate("strips", 120_000, 9))]
    for name, las in inputs:
        assert gpu_ctx.laz_decode(to_laz(las, chunk_size)) == las_records(las), name


@pytest.mark.parametrize("case,method", LAZ_CASES, ids=[f"{c['name']}-{m}" for c, m in LAZ_CASES])
def test_laz_sources_match_pinned_reference(gpu_ctx, case, method):
    conv = gpu_ctx.convert(laz_sources_for(case), method=method, name=case["meta_name"], attributes=case["attributes"])
    assert conv.stats["laz_chunks"] > 0
    for f in FILES:
        exp = case["outputs"][method][f]
        got = _bytes(conv, f)
        assert len(got) == exp["size"], f
        assert md5(got) == exp["md5"], f


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_laz_equals_las(gpu_ctx, method):
    from potreeconverter_b200 import synth
    las = synth.generate("terrain", 400_000, 12)
    a = gpu_ctx.convert(las, method=method, name="t")
    b = gpu_ctx.convert(to_laz(las, 20_000), method=method, name="t")
    assert b.stats["laz_chunks"] == 20
    for f in FILES:
        assert _bytes(a, f) == _bytes(b, f), f


def test_malformed_laz_is_refused(gpu_ctx):
    # corrupted chunk bytes and a file cut short are reported, not decoded
    # past their ends (the decoder's bounds are also fuzzed on the host)
    from potreeconverter_b200 import synth
    import struct
    laz = bytearray(to_laz(synth.generate("hotspots", 30_000, 4), 5000))
    table = struct.unpack_from("<q", laz, struct.unpack_from("<I", laz, 96)[0])[0]
    rng = np.random.default_rng(1)
    refused = 0
    for trial in range(6):
        bad = bytearray(laz)
        lo = struct.unpack_from("<I", laz, 96)[0] + 8 + 200
        for p in rng.integers(lo, table, 6):
            bad[int(p)] ^= 0x5A
        try:
            gpu_ctx.laz_decode(bytes(bad))
        except pc.PcgError as e:
            assert e.status == 1
            refused += 1
    assert refused >= 1
    with pytest.raises(pc.PcgError) as e:
        gpu_ctx.convert(bytes(laz[: len(laz) // 2]))
    assert e.value.status == 1


def test_request_loop_and_cli_take_laz(gpu_ctx, tmp_path):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(200_000, 41)
    lazs = [to_laz(t, 10_000) for t in tiles]
    exp = gpu_ctx.convert(tiles, method="poisson", name="t0")
    got = gpu_ctx.wait(gpu_ctx.submit(lazs, method="poisson", name="t0"))
    for f in FILES:
        assert _bytes(got, f) == _bytes(exp, f), f
    d = tmp_path / "in"
    d.mkdir()
    for k, z in enumerate(lazs):
        (d / f"t{k}.laz").write_bytes(z)
    out = tmp_path / "out"
    exe = os.path.join(os.path.dirname(pc.__file__), "PotreeConverter")
    r = subprocess.run([exe, str(d), "-o", str(out), "-m", "poisson"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    conv = gpu_ctx.convert(tiles, method="poisson", name="in")
    for f in FILES:
        assert (out / f).read_bytes() == _bytes(conv, f), f


def test_laz_decode_throughput(gpu_ctx):
    # 10M points of the hotspots workload (LASzip's default 50,000-point
    # chunks): device decode time per conversion, printed for the record
    from potreeconverter_b200 import synth
    las = synth.generate("hotspots", 10_000_000, 1)
    laz = to_laz(las)
    gpu_ctx.convert_stats(laz)  # warm-up
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        st = gpu_ctx.convert_stats(laz)
        runs.append((time.perf_counter() - t0, st["ms_decode"], st["ms_total"]))
    wall, dec, tot = sorted(runs)[1]
    print(f"\nLAZ 10M hotspots: {len(laz) / 1e6:.0f} MB, {st['laz_chunks']} chunks, decode {dec:.1f} ms "
          f"({10.0 / dec * 1e3:.1f} Mpts/s), conversion {tot:.1f} ms")
    assert st["laz_chunks"] == 200
