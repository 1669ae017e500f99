"""The library's host-side parsers under AddressSanitizer and UBSan, fuzzed
with fixed seeds: the LAZ decoder (the same source the device kernel runs)
on corrupted chunks and chunk tables, and the LAS/LAZ header parsing and
job set-up on mutated headers. Any access outside the inputs, or undefined
behaviour, fails the run."""

import os
import subprocess

import pytest

from tests.oracle_lib import have_laz_tool, to_laz

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "potreeconverter_b200", "csrc")
SAN = ["-std=c++17", "-O1", "-g", "-fsanitize=address,undefined", "-fno-sanitize-recover=all", "-I" + CSRC,
       "-I" + os.path.join(REPO, "include")]


def _build(tmp, name, extra=()):
    exe = str(tmp / name)
    subprocess.run(["g++", *SAN, os.path.join(REPO, "tests", "cpp", name + ".cpp"), *extra, "-o", exe], check=True)
    return exe


def _inputs(tmp):
    from potreeconverter_b200 import synth
    files = []
    for k, img in enumerate(synth.tiles(40_000, 12)):
        p = tmp / f"t{k}.las"
        p.write_bytes(img)
        files.append(p)
    return files


@pytest.mark.skipif(not have_laz_tool(), reason="oracle/_ref/laz_tool not built (make -C oracle ref REF=<reference tree>)")
def test_laz_decoder_under_sanitizers(tmp_path):
    exe = _build(tmp_path, "laz_fuzz")
    for k, las in enumerate(_inputs(tmp_path)):
        laz = tmp_path / f"t{k}.laz"
        laz.write_bytes(to_laz(las.read_bytes(), 2000))
        r = subprocess.run([exe, str(laz), str(11 + k), "150"], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout + r.stderr
        assert "valid decoded 30" in r.stdout, r.stdout


def test_parsers_under_sanitizers(tmp_path):
    exe = _build(tmp_path, "parse_fuzz", [os.path.join(CSRC, "setup.cpp")])
    files = [str(p) for p in _inputs(tmp_path)]
    if have_laz_tool():
        for k in (1, 2):
            z = tmp_path / f"z{k}.laz"
            z.write_bytes(to_laz(open(files[k], "rb").read(), 3000))
            files.append(str(z))
    r = subprocess.run([exe, "5", "6000", *files], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "accepted" in r.stdout
