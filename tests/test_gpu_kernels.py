"""Single-kernel parity: the device replay of std::sort and std::shuffle
against libstdc++ itself (through the oracle library), and the counting
pass (decode, quantization, count grid) against the oracle's."""

import numpy as np
import pytest

import potreeconverter_b200 as pc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 2, 15, 16, 17, 33, 100, 1000, 4097, 32769, 100_000, 1_000_000])
@pytest.mark.parametrize("ties", ["none", "few", "many", "all"])
def test_sort_matches_std_sort(gpu_ctx, oracle, n, ties):
    rng = np.random.default_rng(n * 7 + len(ties))
    if ties == "none":
        keys = rng.random(n)
    elif ties == "few":
        keys = rng.integers(0, max(1, n), n).astype(np.float64)
    elif ties == "many":
        keys = rng.integers(0, 5, n).astype(np.float64)
    else:
        keys = np.zeros(n)
    assert (gpu_ctx.sort_keys(keys) == oracle.sort_perm(keys)).all()


@pytest.mark.parametrize("pattern", ["sorted", "reversed", "organ", "sawtooth"])
@pytest.mark.parametrize("n", [50_000, 400_000])
def test_sort_adversarial_orders(gpu_ctx, oracle, pattern, n):
    i = np.arange(n, dtype=np.float64)
    keys = {"sorted": i, "reversed": i[::-1].copy(), "organ": np.minimum(i, n - i),
            "sawtooth": i % 97}[pattern]
    assert (gpu_ctx.sort_keys(keys) == oracle.sort_perm(keys)).all()


@pytest.mark.parametrize("n", [70_000, 2_000_000])
def test_sort_quantized_distances(gpu_ctx, oracle, n):
    # squared distances of millimetre-quantized points to a box centre: the
    # key distribution of the samplers, with many exact ties
    rng = np.random.default_rng(n)
    q = rng.integers(-20_000, 20_000, (n, 3)).astype(np.float64) * 0.001
    keys = (q * q).sum(axis=1)
    assert (gpu_ctx.sort_keys(keys) == oracle.sort_perm(keys)).all()


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 99, 100, 101, 5000, 9999, 10000])
@pytest.mark.parametrize("seed", [1592614637, 0, 1, 2147483647, 4294967295])
def test_shuffle_matches_std_shuffle(gpu_ctx, oracle, n, seed):
    assert (gpu_ctx.shuffle(n, seed) == oracle.shuffle(n, seed)).all()


@pytest.mark.parametrize("kind,n,seed", [("terrain", 300_000, 3), ("hotspots", 250_000, 4), ("lattice", 200_000, 5),
                                         ("exact", 100_000, 6)])
def test_counting_pass_matches_oracle(gpu_ctx, oracle, kind, n, seed):
    # pcg_kernel_decode_count: quantized X, Y, Z, cells and the count grid
    # of the counting pass, element for element
    from potreeconverter_b200 import synth
    las = synth.generate(kind, n, seed)
    exp = oracle.decode_count(las)
    got = gpu_ctx.decode_count(las)
    for name, a, b in zip(("X", "Y", "Z", "cell", "grid"), got, exp):
        assert a.shape == b.shape and (a.astype(np.int64) == b.astype(np.int64)).all(), name


def test_counting_pass_of_laz_and_out_of_box(gpu_ctx, oracle):
    import struct
    from potreeconverter_b200 import synth
    from tests.oracle_lib import have_laz_tool, to_laz
    las = synth.generate("hotspots", 120_000, 8)
    exp = oracle.decode_count(las)
    if have_laz_tool():
        got = gpu_ctx.decode_count(to_laz(las, 9000))
        for name, a, b in zip(("X", "Y", "Z", "cell", "grid"), got, exp):
            assert (a.astype(np.int64) == b.astype(np.int64)).all(), name
    bad = bytearray(las)
    for off in (179, 195, 211):  # halve the header maxima: points leave the cube
        struct.pack_into("<d", bad, off, struct.unpack_from("<d", bad, off)[0] * 0.5)
    with pytest.raises(pc.PcgError) as e:
        gpu_ctx.decode_count(bytes(bad))
    assert e.value.status == 2
