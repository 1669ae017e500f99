"""The oracle (CPU restatement) is pinned against the reference: its three
output files must match, byte for byte, the digests the pinned reference
converter produced for the same seeded inputs (tests/golden/golden.json)."""

import pytest

from tests.oracle_lib import las_for, load_golden, md5, sources_for

CASES = [(c, m) for c in load_golden()["cases"] for m in c["outputs"]]
MULTI = [(c, m) for c in load_golden()["multi_cases"] for m in c["outputs"]]


@pytest.mark.parametrize("case,method", CASES, ids=[f"{c['name']}-{m}" for c, m in CASES])
def test_oracle_matches_pinned_reference(oracle, case, method):
    out = oracle.convert(las_for(case), method, name=case["name"])
    for f in ("octree.bin", "hierarchy.bin", "metadata.json"):
        assert len(out[f]) == case["outputs"][method][f]["size"], f
        assert md5(out[f]) == case["outputs"][method][f]["md5"], f


@pytest.mark.parametrize("case,method", MULTI, ids=[f"{c['name']}-{m}" for c, m in MULTI])
def test_oracle_sources_and_attributes_match_pinned_reference(oracle, case, method):
    # several LAS files (point formats 0-3, own scales and offsets, extra
    # bytes) and --attributes lists, against the pinned reference
    out = oracle.convert_sources(sources_for(case), method, name=case["meta_name"], attributes=case["attributes"])
    for f in ("octree.bin", "hierarchy.bin", "metadata.json"):
        assert len(out[f]) == case["outputs"][method][f]["size"], f
        assert md5(out[f]) == case["outputs"][method][f]["md5"], f


def test_oracle_rejects_what_the_reference_leaves_undefined(oracle):
    from potreeconverter_b200 import synth
    tiles = synth.tiles(20_000, 3)
    # extra bytes kept while standard attributes before them are dropped:
    # the reference writes them past the point record
    with pytest.raises(RuntimeError, match="past the point record"):
        oracle.convert_sources(tiles, "poisson", attributes=["amplitude"])
    # poisson_average reads rgb at offset -1 when rgb is filtered out
    with pytest.raises(RuntimeError, match="rgb"):
        oracle.convert_sources(tiles[:2], "poisson_average", attributes=["intensity"])


def test_oracle_std_sort_ties_are_deterministic(oracle):
    import numpy as np
    rng = np.random.default_rng(5)
    keys = rng.integers(0, 7, 5000).astype(np.float64)
    p1, p2 = oracle.sort_perm(keys), oracle.sort_perm(keys)
    assert (p1 == p2).all()
    assert (np.diff(keys[p1]) >= 0).all()
    # ties are not in input order: std::sort is not stable
    assert not (p1 == np.argsort(keys, kind="stable")).all()


def test_oracle_shuffle_is_a_permutation(oracle):
    import numpy as np
    for n in (0, 1, 2, 3, 10, 9999, 10000):
        p = oracle.shuffle(n)
        assert sorted(p.tolist()) == list(range(n))


@pytest.mark.parametrize("kind,n,seed", [("terrain", 60_000, 3), ("hotspots", 50_000, 4), ("tiles", 40_000, 5)])
def test_oracle_counting_pass_matches_numpy(oracle, kind, n, seed):
    # the oracle's counting-pass hook against the same FP64 expressions in
    # numpy (chunker_countsort_laszip.cpp:213-257): x = scale X + offset,
    # X' = int32((x - offset') / scale'), cell = ix + iy G + iz G^2
    import struct
    import numpy as np
    from potreeconverter_b200 import synth
    las = synth.generate(kind, n, seed) if kind != "tiles" else synth.tiles(n, seed)[3]
    X, Y, Z, cell, grid = oracle.decode_count(las)
    off = struct.unpack_from("<I", las, 96)[0]
    rl = struct.unpack_from("<H", las, 105)[0]
    cnt = struct.unpack_from("<I", las, 107)[0]
    raw = np.frombuffer(las, dtype=np.dtype({"names": ["X", "Y", "Z"], "formats": ["<i4"] * 3, "offsets": [0, 4, 8],
                                             "itemsize": rl}), count=cnt, offset=off)
    sc = struct.unpack_from("<3d", las, 131)
    of = struct.unpack_from("<3d", las, 155)
    mx = struct.unpack_from("<6d", las, 179)
    hmin = np.array([mx[1], mx[3], mx[5]])
    hmax = np.array([mx[0], mx[2], mx[4]])
    size = hmax - hmin
    pscale = np.maximum(np.array(sc), size / 2.0 ** 30)
    cube = max(size)
    g = 128
    cells = np.zeros(cnt, np.int64)
    for a, (name, q) in enumerate(zip("XYZ", (X, Y, Z))):
        x = sc[a] * raw[name].astype(np.float64) + of[a]
        qq = ((x - hmin[a]) / pscale[a]).astype(np.int32)
        assert (qq == q).all(), name
        u = (qq.astype(np.float64) * pscale[a] + hmin[a] - hmin[a]) / cube
        i = np.minimum(g * u, g - 1.0).astype(np.int64)
        cells += i * g ** a
    assert (cells == cell).all()
    assert (np.bincount(cells, minlength=g ** 3) == grid).all()
