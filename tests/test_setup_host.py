"""The library's job set-up (potreeconverter_b200/csrc/setup.cpp), built for
the host: for several sources and --attributes lists it yields the output
schema, scale, offset and cube the oracle (pinned to the reference) writes
into metadata.json; extra bytes are placed by the reference's rule; LAZ
headers and chunk tables are read; lists whose result the reference leaves
undefined are refused. No GPU is involved."""

import json
import os
import re
import subprocess

import pytest

from tests.oracle_lib import have_laz_tool, to_laz

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "potreeconverter_b200", "csrc")


@pytest.fixture(scope="module")
def setup_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("setup") / "setup_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I" + CSRC, "-I" + os.path.join(REPO, "include"),
                    os.path.join(REPO, "tests", "cpp", "setup_check.cpp"), os.path.join(CSRC, "setup.cpp"), "-o", exe],
                   check=True)
    return exe


def _run(exe, tmp_path, images, attributes=()):
    paths = []
    for k, img in enumerate(images):
        paths.append(str(tmp_path / f"s{k}.las"))
        with open(paths[-1], "wb") as f:
            f.write(img)
    cmd = [exe] + paths + (["--attributes"] + list(attributes) if attributes else [])
    return json.loads(subprocess.run(cmd, check=True, capture_output=True, text=True).stdout)


def _inputs():
    from potreeconverter_b200 import synth
    t = synth.tiles(40_000, 5)
    h = synth.generate("hotspots", 30_000, 6)
    return [
        ("tiles", t, []),
        ("tiles reversed", t[::-1], []),
        ("tiles filtered", t, ["gps-time", "rgb", "return number", "no such"]),
        ("formats 1 and 2", [t[3], t[0]], ["intensity", "classification"]),
        ("hotspots reordered", [h], ["extra", "intensity", "return number", "number of returns", "classification",
                                     "scan angle rank", "user data", "point source id", "gps-time", "rgb"]),
        ("empty source", synth.sources("tiles_empty", 40_000, 7), []),
    ]


@pytest.mark.parametrize("idx", range(6))
def test_schema_matches_oracle_metadata(setup_check, oracle, tmp_path, idx):
    name, images, attrs = _inputs()[idx]
    got = _run(setup_check, tmp_path, images, attrs)
    # the reference writes non-finite statistics as inf
    text = oracle.convert_sources(images, "random", attributes=attrs)["metadata.json"].decode()
    md = json.loads(re.sub(r"(?<![A-Za-z])(-?)inf(?![A-Za-z])", r"\1Infinity", text))
    assert [(a["name"], a["size"]) for a in got["attributes"]] == [(a["name"], a["size"]) for a in md["attributes"]], name
    assert got["bpp"] == sum(a["size"] for a in md["attributes"])
    assert got["points"] == md["points"]
    assert got["scale"] == md["scale"] and got["offset"] == md["offset"], name
    assert got["min"] == md["boundingBox"]["min"] and got["max"] == md["boundingBox"]["max"], name
    assert [a["type"] for a in got["attributes"]] == [a["type"] for a in md["attributes"]]


def test_extra_bytes_follow_the_reference_rule(setup_check, tmp_path):
    # a kept extra goes to its source's standard size plus the sizes of the
    # kept extras before it (chunker_countsort_laszip.cpp:565-653)
    from potreeconverter_b200 import synth
    t = synth.tiles(20_000, 8)
    got = _run(setup_check, tmp_path, t)
    std = {2: 27, 0: 21, 3: 35, 1: 29}  # position .. point source id, + gps-time (8), + rgb (6)
    sizes = {a["name"]: a["size"] for a in got["attributes"]}
    index = {a["name"]: i for i, a in enumerate(got["attributes"])}
    for fmt, names, src in zip(synth.TILE_FORMATS, synth.TILE_EXTRAS, got["sources"]):
        dst = std[fmt]
        expect = []
        src_off = {0: 20, 1: 28, 2: 26, 3: 34}[fmt]
        for n in names:
            expect.append([src_off, dst, sizes[n], index[n]])
            dst += sizes[n]
            src_off += sizes[n]
        assert src["extras"] == expect, fmt


@pytest.mark.skipif(not have_laz_tool(), reason="oracle/_ref/laz_tool not built (make -C oracle ref REF=<reference tree>)")
def test_laz_sources_are_read(setup_check, tmp_path):
    from potreeconverter_b200 import synth
    t = synth.tiles(40_000, 9)
    las_view = _run(setup_check, tmp_path, t)
    laz_view = _run(setup_check, tmp_path, [to_laz(t[0], 3000), t[1], to_laz(t[2], 0), t[3]])
    for k in ("bpp", "points", "scale", "offset", "min", "max", "attributes"):
        assert laz_view[k] == las_view[k], k
    s = laz_view["sources"]
    assert [x["compressed"] for x in s] == [True, False, True, False]
    assert s[0]["laz_chunks"] == -(-s[0]["points"] // 3000) and s[2]["laz_chunks"] == 1


def test_undefined_lists_are_refused(setup_check, tmp_path):
    from potreeconverter_b200 import synth
    t = synth.tiles(20_000, 3)
    for attrs, msg in ((["amplitude"], "past the point record"), (["rgb", "rgb"], "twice"), (["position"], "twice")):
        got = _run(setup_check, tmp_path, t, attrs)
        assert msg in got.get("error", ""), attrs


def test_malformed_headers_are_refused(setup_check, tmp_path):
    # counts that overflow the size arithmetic, truncated records, and a LAZ
    # chunk table that claims more chunks than points are errors, not crashes
    import struct
    from potreeconverter_b200 import synth
    las = bytearray(synth.generate("hotspots", 5_000, 2))  # LAS 1.4: 64-bit point count at 247
    cases = []
    big = bytearray(las)
    struct.pack_into("<Q", big, 247, (1 << 63) + 5)
    cases.append((bytes(big), "implausible point count"))
    wrap = bytearray(las)
    struct.pack_into("<Q", wrap, 247, (1 << 64) // struct.unpack_from("<H", las, 105)[0] + 1)
    cases.append((bytes(wrap), "point count"))
    cases.append((bytes(las[: len(las) - 100]), "truncated point data"))
    if have_laz_tool():
        laz = bytearray(to_laz(bytes(las), 1000))
        table = struct.unpack_from("<q", laz, struct.unpack_from("<I", laz, 96)[0])[0]
        struct.pack_into("<I", laz, table + 4, 10_000)  # 10,000 chunks for 5,000 points
        cases.append((bytes(laz), "chunk table"))
    for img, msg in cases:
        got = _run(setup_check, tmp_path, [img])
        assert msg in got.get("error", ""), (msg, got)
