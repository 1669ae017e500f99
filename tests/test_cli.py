"""The PotreeConverter command line's argument handling, up to the point
where it opens a device (no GPU needed): the reference's flags, its exit
code 123 for a missing input, refusals of what this build does not do."""

import os
import subprocess

import pytest

import potreeconverter_b200 as pc

EXE = os.path.join(os.path.dirname(pc.__file__), "PotreeConverter")
pytestmark = pytest.mark.skipif(not os.path.exists(EXE), reason="command line not built")


def _run(*args, cwd=None):
    return subprocess.run([EXE, *args], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_help_and_usage():
    assert _run("--help").returncode == 0
    r = _run()
    assert r.returncode == 1 and "PotreeConverter <source>" in r.stderr


def test_missing_source_exits_123(tmp_path):
    # main.cpp:81-85: a first source that does not exist ends with exit(123)
    r = _run(str(tmp_path / "nothing.las"), "-o", str(tmp_path / "out"))
    assert r.returncode == 123 and "does not exist" in r.stderr


def test_refused_flags(tmp_path):
    src = tmp_path / "a.las"
    src.write_bytes(b"x")
    for args, msg in ((["--encoding", "BROTLI"], "not supported"), (["-m", "nearest"], "unknown method"),
                      (["--generate-page", "p"], "not supported"), (["--keep-chunks"], "not supported"),
                      (["--chunkMethod", "OTHER"], "LASZIP"), (["--frobnicate"], "unknown flag")):
        r = _run(str(src), "-o", str(tmp_path / "out"), *args)
        assert r.returncode == 1 and msg in r.stderr, args


def test_directory_without_las_files(tmp_path):
    d = tmp_path / "empty"
    d.mkdir()
    (d / "readme.txt").write_text("no point clouds here")
    r = _run(str(d), "-o", str(tmp_path / "out"))
    assert r.returncode == 1 and "no LAS input" in r.stderr
