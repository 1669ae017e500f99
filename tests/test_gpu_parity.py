"""End-to-end parity through the C ABI: octree.bin, hierarchy.bin and
metadata.json written by the CUDA pipeline are byte-identical to the
pinned reference's (golden digests) and to the oracle, for every sampler,
in both the batched and the plain form."""

import pytest

import potreeconverter_b200 as pc
from tests.oracle_lib import las_for, load_golden, md5

pytestmark = pytest.mark.gpu

CASES = [(c, m) for c in load_golden()["cases"] for m in c["outputs"]]
FILES = {"octree.bin": "octree", "hierarchy.bin": "hierarchy", "metadata.json": "metadata"}


def _bytes(conv, f):
    v = getattr(conv, FILES[f])
    return v.encode() if isinstance(v, str) else v


@pytest.mark.parametrize("case,method", CASES, ids=[f"{c['name']}-{m}" for c, m in CASES])
def test_batched_matches_pinned_reference(gpu_ctx, case, method):
    conv = gpu_ctx.convert(las_for(case), method=method, name=case["name"])
    for f in FILES:
        got = _bytes(conv, f)
        exp = case["outputs"][method][f]
        assert len(got) == exp["size"], f
        assert md5(got) == exp["md5"], f


@pytest.mark.parametrize("case,method", [(c, m) for c, m in CASES if c["points"] <= 300_000],
                         ids=[f"{c['name']}-{m}" for c, m in CASES if c["points"] <= 300_000])
def test_plain_form_matches_pinned_reference(case, method):
    with pc.Context(form="plain") as ctx:
        conv = ctx.convert(las_for(case), method=method, name=case["name"])
    for f in FILES:
        assert md5(_bytes(conv, f)) == case["outputs"][method][f]["md5"], f


@pytest.mark.parametrize("kind,n,seed", [("terrain", 600_000, 31), ("hotspots", 400_000, 32),
                                         ("lattice", 800_000, 33), ("strips", 500_000, 34)])
@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_matches_oracle_on_fresh_inputs(gpu_ctx, oracle, kind, n, seed, method):
    from potreeconverter_b200 import synth
    las = synth.generate(kind, n, seed)
    exp = oracle.convert(las, method, name="fresh")
    conv = gpu_ctx.convert(las, method=method, name="fresh")
    for f in FILES:
        assert _bytes(conv, f) == exp[f], f


@pytest.mark.parametrize("method", ["poisson", "poisson_average"])
def test_cluster_acceptance_matches_oracle(gpu_ctx, oracle, method):
    # a volumetric cloud: its upper nodes hold enough candidates to be
    # accepted by a cluster of CTAs (at least 65,536 candidates per node)
    from potreeconverter_b200 import synth
    las = synth.generate("cube", 400_000, 41)
    exp = oracle.convert(las, method, name="cube")
    conv = gpu_ctx.convert(las, method=method, name="cube")
    assert conv.stats["cluster_nodes"] > 0
    for f in FILES:
        assert _bytes(conv, f) == exp[f], f


def test_out_of_box_point_is_reported(gpu_ctx):
    from potreeconverter_b200 import synth
    import struct
    las = bytearray(synth.terrain(5000, 9))
    # the reference checks points against the cubic box min + max extent
    # (chunker_countsort_laszip.cpp:205-251): halving every header maximum
    # halves the cube, and points beyond it must be reported
    for off in (179, 195, 211):
        struct.pack_into("<d", las, off, struct.unpack_from("<d", las, off)[0] * 0.5)
    with pytest.raises(pc.PcgError) as e:
        gpu_ctx.convert(bytes(las))
    assert e.value.status in (2,)


def test_bad_input_is_rejected(gpu_ctx):
    with pytest.raises(pc.PcgError) as e:
        gpu_ctx.convert(b"not a las file at all" * 20)
    assert e.value.status == 1


@pytest.mark.parametrize("method", ["poisson", "poisson_average", "random"])
def test_node_records_match_oracle(gpu_ctx, oracle, method):
    # pcg_result.nodes: every node in completion order with its payload's
    # place in octree.bin, as the reference's hierarchy flusher records them
    from potreeconverter_b200 import synth
    las = synth.generate("terrain", 300_000, 21)
    exp = oracle.convert(las, method, name="n")["nodes"]
    conv = gpu_ctx.convert(las, method=method, name="n")
    assert conv.nodes == exp
    assert len(conv.nodes) == conv.stats["num_nodes"]
    assert sum(n[2] for n in conv.nodes) == len(conv.octree)
