"""The oracle's stage hooks (pcref_lut, pcref_scatter, pcref_octree,
pcref_accept), which the stage-level GPU tests compare against, pinned to
the oracle's whole conversion (itself pinned to the reference's digests):
the chunk list and point counts, the octree's node names, and one node's
acceptance restated here in plain Python for small inputs."""

import json
import math

import numpy as np
import pytest

from tests.oracle_lib import case_las
from tests.stage_inputs import StageInputs

CLOUDS = [("terrain", 60_000, 1000, {}), ("hotspots", 80_000, 1001, {}), ("lattice", 60_000, 1002, {"cube": 128.0})]


@pytest.fixture(scope="module", params=CLOUDS, ids=[c[0] for c in CLOUDS])
def cloud(request, oracle):
    kind, n, seed, kw = request.param
    las = case_las(kind, n, seed, json.dumps(kw, sort_keys=True))
    return StageInputs(oracle, las), oracle.convert(las, "poisson")


def test_lut_and_scatter_hooks_match_conversion(cloud):
    st, conv = cloud
    assert [(c[0], c[5]) for c in st.chunks] == conv["chunks"]
    assert list(np.diff(st.chunk_start)) == [c for _, c in conv["chunks"]]
    for k in range(len(st.chunks)):
        seg = st.ids[st.chunk_start[k]: st.chunk_start[k + 1]]
        assert (np.diff(seg.astype(np.int64)) > 0).all()  # input order inside a chunk
    # every cell of the grid with points is covered by a chunk
    assert (st.lut[st.cell] >= 0).all()


def test_octree_hook_matches_conversion_nodes(cloud, oracle):
    st, conv = cloud
    names = {n[0] for n in conv["nodes"]}
    for k in st.largest_chunks(2):
        X, Y, Z, name, bmin, bmax = st.chunk_points(k)
        order, nodes, _ = oracle.octree(X, Y, Z, st.scale, st.offset, bmin, bmax, name)
        got = {nm for nm, _, _, _ in nodes if nm != name}
        # poisson completes every node below a chunk root (App. A6)
        assert got == {nm for nm in names if nm.startswith(name) and nm != name}
        kept = sum(c for _, _, c, _ in nodes)
        assert sorted(order[:kept].tolist()) == list(range(kept)) or kept < X.shape[0]


def _poisson_py(x, y, z, ctr, spacing, perm):
    """sampler_poisson.h:127-180 for a small node: candidates in std::sort
    order (perm), newest accepted first, early exit, 10,001-check cap."""
    acc = []
    out = np.zeros(x.shape[0], np.uint8)
    s2 = spacing * spacing
    for i in perm:
        cx, cy, cz = x[i] - ctr[0], y[i] - ctr[1], z[i] - ctr[2]
        cd = math.sqrt(cx * cx + cy * cy + cz * cz)
        lim = (cd - spacing) * (cd - spacing)
        ok, j = True, 0
        for a in reversed(acc):
            px, py, pz = x[a] - ctr[0], y[a] - ctr[1], z[a] - ctr[2]
            if px * px + py * py + pz * pz < lim:
                break
            dx, dy, dz = x[a] - x[i], y[a] - y[i], z[a] - z[i]
            if dx * dx + dy * dy + dz * dz < s2:
                ok = False
                break
            j += 1
            if j > 10_000:
                break
        if ok:
            acc.append(i)
            out[i] = 1
    return out


def _random_py(x, y, z, child, bmin, bmax):
    """sampler_random.h:123-182 for the first node a thread samples."""
    G = 128
    size = bmax - bmin
    taken = set()
    out = np.zeros(x.shape[0], np.uint8)
    counts = np.bincount(child, minlength=8)
    for i in range(x.shape[0]):
        n = [(x[i] - bmin[0]) / size[0], (y[i] - bmin[1]) / size[1], (z[i] - bmin[2]) / size[2]]
        loc = [2.0 * math.fmod(G * v, 1.0) - 1.0 for v in n]
        dist = math.sqrt(sum(v * v for v in loc))
        cell = tuple(max(0, min(int(G * v), G - 1)) for v in n)
        if counts[child[i]] < 100 or (dist < 0.7 * math.sqrt(3.0) and cell not in taken):
            out[i] = 1
            taken.add(cell)
    return out


def test_accept_hook_matches_python_restatement(cloud, oracle):
    st, _ = cloud
    X, Y, Z, child, bmin, bmax, spacing = st.node_candidates(st.X[:3000], st.Y[:3000], st.Z[:3000], "r")
    x = X * st.scale[0] + st.offset[0]
    y = Y * st.scale[1] + st.offset[1]
    z = Z * st.scale[2] + st.offset[2]
    for sp in (spacing, spacing * 0.05):
        ctr = (bmin + bmax) * 0.5
        keys = (x - ctr[0]) ** 2 + (y - ctr[1]) ** 2 + (z - ctr[2]) ** 2
        exp = _poisson_py(x, y, z, ctr, sp, oracle.sort_perm(keys))
        got, _ = oracle.accept("poisson", X, Y, Z, child, st.scale, st.offset, bmin, bmax, sp)
        assert (got == exp).all()
    got, _ = oracle.accept("random", X, Y, Z, child, st.scale, st.offset, bmin, bmax, spacing)
    assert (got == _random_py(x, y, z, child, bmin, bmax)).all()
