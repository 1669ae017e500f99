"""pcg_kernel_sort_keys_noalloc -- the std::sort replay for callers that
cannot allocate device memory: a plugin inside a host framework that owns
every device allocation and hands its plugins only the buffers it made. Its
scratch is a static device array; inputs and outputs are the caller's device
buffers.

Each case is checked on two calls in a row (the second call reuses the array
the first one left behind) against the allocating entry point,
pcg_kernel_sort_keys, and against libstdc++'s std::sort run by the oracle.
Permutations must match exactly. Sizes cover one key, a single insertion-sort
block, both sides of the switch from one warp to a whole CTA (4,095 / 4,096
keys) and the maximum, with random keys, all-equal keys and few distinct
values. Kept in its own file, collected last, so a failure here stops a -x
run only after every other test ran."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX = 262144  # PCG_NOALLOC_SORT_MAX in include/pcgpu.h


def _noalloc_sort(lib, keys):
    import torch
    d_keys = torch.from_numpy(np.ascontiguousarray(keys, dtype=np.float64)).cuda()
    d_perm = torch.full((keys.shape[0],), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    st = lib.pcg_kernel_sort_keys_noalloc(d_keys.data_ptr(), keys.shape[0], d_perm.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    return st, d_perm.cpu().numpy(), free0 - free1


def _keys(kind, n, rng):
    if kind == "random":
        return rng.random(n)
    if kind == "equal":
        return np.full(n, 2.5)
    return rng.integers(0, 9, n).astype(np.float64)  # few distinct values: long runs of ties


@pytest.mark.parametrize("n", [1, 17, 4095, 4096, MAX])
@pytest.mark.parametrize("kind", ["random", "equal", "ties"])
def test_noalloc_sort_matches_std_sort_twice(n, kind):
    import potreeconverter_b200 as pc
    from tests.oracle_lib import Oracle
    lib = pc.load_library()
    rng = np.random.default_rng(2024 + n)
    oracle = Oracle()
    with pc.Context() as ctx:
        # the first calls of the process load the module holding the array
        # and the code of both sort kernels (one warp, one CTA)
        _noalloc_sort(lib, np.zeros(8))
        _noalloc_sort(lib, np.zeros(4096))
        for call in range(2):
            keys = _keys(kind, n, rng)
            st, perm, used = _noalloc_sort(lib, keys)
            assert st == 0, f"call {call}: status {st}"
            assert (perm == oracle.sort_perm(keys)).all(), f"call {call}: differs from std::sort"
            assert (perm == ctx.sort_keys(keys)).all(), f"call {call}: differs from the allocating entry point"
            assert used == 0, f"call {call}: device memory fell by {used} bytes"


def test_noalloc_sort_rejects_oversize_input():
    import potreeconverter_b200 as pc
    lib = pc.load_library()
    assert lib.pcg_kernel_sort_keys_noalloc(None, MAX + 1, None, None) == 1  # PCG_BAD_INPUT
