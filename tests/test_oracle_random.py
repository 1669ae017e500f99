"""The oracle against the pinned reference binary itself (oracle/_ref/
PotreeConverter_pinned, built from the reference sources by oracle/Makefile)
on seeded random jobs beyond the golden cases: random subsets and orders of
tiles in point formats 0-3, random --attributes lists whose result the
reference defines, every sampler. Runs where the reference was built."""

import os
import subprocess

import numpy as np
import pytest

from tests.oracle_lib import ORACLE_DIR

REF = os.path.join(ORACLE_DIR, "_ref", "PotreeConverter_pinned")
STANDARD = ["intensity", "return number", "number of returns", "classification", "scan angle rank", "user data",
            "point source id", "gps-time", "rgb"]

pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="pinned reference not built (make -C oracle ref REF=<reference tree>)")


@pytest.mark.parametrize("seed", range(16))
def test_oracle_matches_reference_on_random_jobs(oracle, tmp_path, seed):
    from potreeconverter_b200 import synth
    rng = np.random.default_rng(500 + seed)
    tiles = synth.tiles(int(rng.integers(20_000, 60_000)), 600 + seed)
    order = [int(k) for k in rng.permutation(4)][: int(rng.integers(1, 5))]
    method = ["poisson", "poisson_average", "random"][seed % 3]
    if method == "poisson_average" and not any(synth.TILE_FORMATS[k] in (2, 3) for k in order):
        # without rgb the reference's poisson_average reads and writes at
        # offset -1 (it aborts with heap corruption); the library refuses it
        order.append(0)
    srcs = [tiles[k] for k in order]
    attrs = []
    if seed % 2:
        # standard attributes only: kept extras would land past the record
        attrs = [STANDARD[int(k)] for k in rng.permutation(len(STANDARD))][: int(rng.integers(1, len(STANDARD) + 1))]
        if method == "poisson_average" and "rgb" not in attrs:
            attrs.append("rgb")
    paths = []
    for k, img in zip(order, srcs):
        paths.append(str(tmp_path / f"t{k}.las"))
        with open(paths[-1], "wb") as f:
            f.write(img)
    out = tmp_path / "out"
    cmd = [REF] + paths + ["-o", str(out), "-m", method] + (["--attributes"] + attrs if attrs else [])
    subprocess.run(cmd, check=True, capture_output=True)
    exp = oracle.convert_sources(srcs, method, name=f"t{order[0]}", attributes=attrs)
    for f in ("octree.bin", "hierarchy.bin", "metadata.json"):
        assert (out / f).read_bytes() == exp[f], (f, order, method, attrs)


@pytest.mark.parametrize("seed", range(12))
def test_oracle_matches_reference_on_random_clouds(oracle, tmp_path, seed):
    from potreeconverter_b200 import synth
    rng = np.random.default_rng(700 + seed)
    kind = ["terrain", "hotspots", "lattice", "strips", "duplicates", "cube"][seed % 6]
    n = int(rng.integers(5_000, 80_000))
    las = synth.generate(kind, n, 800 + seed)
    method = ["poisson", "poisson_average", "random"][int(rng.integers(0, 3))]
    path = tmp_path / "cloud.las"
    path.write_bytes(las)
    out = tmp_path / "out"
    subprocess.run([REF, str(path), "-o", str(out), "-m", method], check=True, capture_output=True)
    exp = oracle.convert(las, method, name="cloud")
    for f in ("octree.bin", "hierarchy.bin", "metadata.json"):
        assert (out / f).read_bytes() == exp[f], (f, kind, n, method)


@pytest.mark.skipif(not os.path.exists(os.path.join(ORACLE_DIR, "_ref", "laz_tool")), reason="laz_tool not built")
@pytest.mark.parametrize("seed", range(6))
def test_reference_reads_laz_like_las(oracle, tmp_path, seed):
    # the reference converts LAZ files (written by its own LASzip, random
    # chunk sizes) to the same files as the LAS files they came from, which
    # is what pins LAZ parity to the restatement
    from potreeconverter_b200 import synth
    from tests.oracle_lib import to_laz
    rng = np.random.default_rng(900 + seed)
    tiles = synth.tiles(int(rng.integers(20_000, 60_000)), 950 + seed)
    order = [int(k) for k in rng.permutation(4)][: int(rng.integers(1, 5))]
    method = ["poisson", "poisson_average", "random"][seed % 3]
    if method == "poisson_average" and not any(synth.TILE_FORMATS[k] in (2, 3) for k in order):
        order.append(0)
    paths = []
    for k in order:
        if rng.uniform() < 0.6:
            paths.append(tmp_path / f"t{k}.laz")
            paths[-1].write_bytes(to_laz(tiles[k], int(rng.choice([0, 700, 5000, 33333]))))
        else:
            paths.append(tmp_path / f"t{k}.las")
            paths[-1].write_bytes(tiles[k])
    out = tmp_path / "out"
    subprocess.run([REF] + [str(p) for p in paths] + ["-o", str(out), "-m", method], check=True, capture_output=True)
    exp = oracle.convert_sources([tiles[k] for k in order], method, name=f"t{order[0]}")
    for f in ("octree.bin", "hierarchy.bin", "metadata.json"):
        assert (out / f).read_bytes() == exp[f], (f, [p.name for p in paths], method)
