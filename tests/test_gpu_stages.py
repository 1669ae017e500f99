"""Stage-level parity: the library's entry points for the LUT merge
(pcg_kernel_lut), the distribution to chunks (pcg_kernel_scatter), one
chunk's octree (pcg_kernel_octree) and one node's sampler decision
(pcg_kernel_accept) against the oracle's hooks for the same stage, on the
same arrays, element for element. Inputs come from terrain, hot-spot,
jittered-lattice and exact-arithmetic clouds (tests/stage_inputs.py)."""

import json

import numpy as np
import pytest

from tests.oracle_lib import case_las
from tests.stage_inputs import StageInputs

pytestmark = pytest.mark.gpu

CLOUDS = [("terrain", 200_000, 1000, {}), ("hotspots", 300_000, 1001, {}), ("lattice", 200_000, 1002, {"cube": 128.0}),
          ("exact", 200_000, 3, {})]


@pytest.fixture(scope="module", params=CLOUDS, ids=[c[0] for c in CLOUDS])
def stage(request, oracle):
    kind, n, seed, kw = request.param
    return StageInputs(oracle, case_las(kind, n, seed, json.dumps(kw, sort_keys=True)))


def _same_chunks(got, exp):
    # element by element, reporting the first difference (a plain list
    # comparison of 10^5 chunks makes pytest's failure diff very slow)
    assert len(got) == len(exp), f"{len(got)} chunks, expected {len(exp)}"
    bad = next((i for i, (a, b) in enumerate(zip(got, exp)) if a != b), None)
    assert bad is None, f"chunk {bad}: {got[bad]} != {exp[bad]}"


def _same_lut(got, exp):
    bad = np.nonzero(got != exp)[0]
    assert bad.size == 0, f"{bad.size} LUT cells differ, first {bad[0]}: {got[bad[0]]} != {exp[bad[0]]}"


def test_lut_matches_oracle(gpu_ctx, stage):
    chunks, lut = gpu_ctx.lut(stage.grid, stage.G, stage.mpc)
    _same_chunks(chunks, stage.chunks)
    _same_lut(lut, stage.lut)


@pytest.mark.parametrize("mpc", [1, 5_000, 10**9])
def test_lut_merge_limits(gpu_ctx, oracle, stage, mpc):
    # every cell its own chunk, a mid-size limit, and one chunk for all
    exp_chunks, exp_lut = oracle.lut(stage.grid, stage.G, mpc)
    chunks, lut = gpu_ctx.lut(stage.grid, stage.G, mpc)
    _same_chunks(chunks, exp_chunks)
    _same_lut(lut, exp_lut)


def test_scatter_matches_oracle(gpu_ctx, stage):
    ids, start = gpu_ctx.scatter(stage.cell, stage.lut, stage.G, len(stage.chunks))
    assert np.array_equal(start, stage.chunk_start)
    assert np.array_equal(ids, stage.ids)


def test_scatter_empty_and_reversed(gpu_ctx, oracle, stage):
    ids, start = gpu_ctx.scatter(stage.cell[:0], stage.lut, stage.G, len(stage.chunks))
    assert ids.shape[0] == 0 and (start == 0).all()
    cell = stage.cell[::-1].copy()
    exp_ids, exp_start = oracle.scatter(cell, stage.lut, len(stage.chunks))
    ids, start = gpu_ctx.scatter(cell, stage.lut, stage.G, len(stage.chunks))
    assert (start == exp_start).all() and (ids == exp_ids).all()


def _same_octree(got, exp, what):
    # the same nodes (name, point count, leaf or not), the same depth, and
    # every leaf's points in the same order; where a leaf starts in the
    # order array may differ (points the duplicate rule drops stay in the
    # library's array)
    assert [(n, c, lf) for n, _, c, lf in got[1]] == [(n, c, lf) for n, _, c, lf in exp[1]], f"{what}: node list differs"
    assert got[2] == exp[2], f"{what}: octree depth differs"
    for (name, gs, c, lf), (_, es, _, _) in zip(got[1], exp[1]):
        if lf and c:
            assert (got[0][gs:gs + c] == exp[0][es:es + c]).all(), f"{what}: points of {name} differ"


def test_octree_matches_oracle(gpu_ctx, oracle, stage):
    for k in stage.largest_chunks(3):
        X, Y, Z, name, bmin, bmax = stage.chunk_points(k)
        exp = oracle.octree(X, Y, Z, stage.scale, stage.offset, bmin, bmax, name)
        got = gpu_ctx.octree(X, Y, Z, stage.scale, stage.offset, bmin, bmax, name)
        _same_octree(got, exp, f"chunk {name}")


def test_octree_whole_cloud_as_one_chunk(gpu_ctx, oracle, stage):
    # the whole cloud in one node: deep recursion, duplicate rule where the
    # input has coincident points
    exp = oracle.octree(stage.X, stage.Y, stage.Z, stage.scale, stage.offset, stage.cube_min,
                        stage.cube_min + stage.cube_size, "r")
    got = gpu_ctx.octree(stage.X, stage.Y, stage.Z, stage.scale, stage.offset, stage.cube_min,
                         stage.cube_min + stage.cube_size, "r")
    _same_octree(got, exp, "whole cloud")


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_accept_matches_oracle(gpu_ctx, oracle, stage, method):
    rng = np.random.default_rng(5)
    cases = []
    # the root over the first 40,000 points, and the cubes of the two
    # largest chunks (the oracle decides a node's candidates one by one)
    cases.append(stage.node_candidates(stage.X[:40_000], stage.Y[:40_000], stage.Z[:40_000], "r"))
    for k in stage.largest_chunks(2):
        X, Y, Z, name, _, _ = stage.chunk_points(k)
        cases.append(stage.node_candidates(X, Y, Z, name))
    for X, Y, Z, child, bmin, bmax, spacing in cases:
        rgb = rng.integers(0, 65536, (X.shape[0], 3), dtype=np.uint16) if method == "poisson_average" else None
        exp_acc, exp_rgb = oracle.accept(method, X, Y, Z, child, stage.scale, stage.offset, bmin, bmax, spacing, rgb)
        got_acc, got_rgb = gpu_ctx.accept(method, X, Y, Z, child, stage.scale, stage.offset, bmin, bmax, spacing, rgb)
        mismatches = int((got_acc != exp_acc).sum())
        assert mismatches == 0, f"{mismatches} acceptance mismatches of {X.shape[0]} candidates"
        if method == "poisson_average":
            assert (got_rgb == exp_rgb).all()


def test_accept_small_and_refused_inputs(gpu_ctx, oracle, stage):
    # one candidate, a child of fewer than 100 points for random, and an
    # unordered child list, which is refused
    X, Y, Z, child, bmin, bmax, spacing = stage.node_candidates(stage.X[:150], stage.Y[:150], stage.Z[:150], "r")
    for method in ("poisson", "random"):
        for m in (1, 150):
            exp = oracle.accept(method, X[:m], Y[:m], Z[:m], child[:m], stage.scale, stage.offset, bmin, bmax, spacing)[0]
            got = gpu_ctx.accept(method, X[:m], Y[:m], Z[:m], child[:m], stage.scale, stage.offset, bmin, bmax, spacing)[0]
            assert (got == exp).all()
    bad = child.copy()
    bad[0], bad[-1] = 7, 0
    import potreeconverter_b200 as pc
    with pytest.raises(pc.PcgError):
        gpu_ctx.accept("poisson", X, Y, Z, bad, stage.scale, stage.offset, bmin, bmax, spacing)
