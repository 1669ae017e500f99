"""The library's LAZ decoder (potreeconverter_b200/csrc/laz.cuh), built for
the host, reproduces the point records LASzip writes: LAZ files made by the
reference's vendored LASzip (oracle/_ref/laz_tool) from seeded LAS files in
point formats 0-3, with and without extra bytes, at several chunk sizes,
decode to the LAS records byte for byte. The device kernel runs the same
code (tests/test_gpu_laz.py)."""

import os
import subprocess

import numpy as np
import pytest

from tests.oracle_lib import have_laz_tool, las_records, to_laz

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.skipif(not have_laz_tool(), reason="oracle/_ref/laz_tool not built (make -C oracle ref REF=<reference tree>)")


@pytest.fixture(scope="module")
def laz_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("laz") / "laz_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(REPO, "potreeconverter_b200", "csrc"),
                    os.path.join(REPO, "tests", "cpp", "laz_check.cpp"), "-o", exe], check=True)
    return exe


def _decode(laz_check, tmp_path, laz: bytes) -> bytes:
    src, dst = tmp_path / "in.laz", tmp_path / "out.bin"
    src.write_bytes(laz)
    r = subprocess.run([laz_check, str(src), str(dst)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return dst.read_bytes()


def _inputs():
    from potreeconverter_b200 import synth
    out = [(f"tile{k}", t) for k, t in enumerate(synth.tiles(120_000, 77))]  # formats 2, 0, 3, 1; extras on 3 and 1
    out += [("hotspots", synth.generate("hotspots", 80_000, 5)), ("lattice", synth.generate("lattice", 60_000, 8))]
    return out


@pytest.mark.parametrize("chunk_size", [0, 1000, 7777])
def test_host_decoder_matches_laszip(laz_check, tmp_path, chunk_size):
    for name, las in _inputs():
        assert _decode(laz_check, tmp_path, to_laz(las, chunk_size)) == las_records(las), name


def test_host_decoder_gps_time_paths(laz_check, tmp_path):
    # interleaved time sequences, repeats and jumps reach every GPS code path
    from potreeconverter_b200 import synth
    rng = np.random.default_rng(3)
    n = 60_000
    X = rng.integers(0, 10**6, n).astype(np.int32)
    Y = rng.integers(0, 10**6, n).astype(np.int32)
    Z = rng.integers(0, 10**5, n).astype(np.int32)
    attrs = synth._common_attrs(rng, n, Z.astype(np.float64))
    seq = rng.integers(0, 4, n)
    base = np.array([1.0e5, 3.0e8, -5.0e3, 7.7e11])
    step = np.array([1e-5, 3.3e-3, 0.5, 123.0])
    t = base[seq] + np.cumsum(np.where(rng.uniform(0, 1, n) < 0.2, 0.0, step[seq]))
    jump = rng.uniform(0, 1, n) < 0.01
    t[jump] = rng.uniform(-1e12, 1e12, int(jump.sum()))
    attrs["gps_time"] = t
    las = synth.write_las(X, Y, Z, attrs, pdrf=3, version_minor=4)
    for cs in (0, 997):
        assert _decode(laz_check, tmp_path, to_laz(las, cs)) == las_records(las)
