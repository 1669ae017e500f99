"""pcg_kernel_sort_keys_noalloc -- the std::sort replay for callers that
cannot allocate device memory (a plugin whose host owns every device
allocation, or code enqueuing work during stream capture). Its scratch is a
static device array; inputs and outputs are the caller's device buffers.

Checked against the allocating entry point, pcg_kernel_sort_keys, on two
calls in a row (the second call reuses the array the first one left
behind). Permutations must match exactly. Kept in its own file, collected
last, so a failure here stops a -x run only after every other test ran."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX = 262144  # PCG_NOALLOC_SORT_MAX in include/pcgpu.h


def _noalloc_sort(lib, keys):
    import torch
    d_keys = torch.from_numpy(np.ascontiguousarray(keys, dtype=np.float64)).cuda()
    d_perm = torch.full((keys.shape[0],), -1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    st = lib.pcg_kernel_sort_keys_noalloc(d_keys.data_ptr(), keys.shape[0], d_perm.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    return st, d_perm.cpu().numpy()


def test_noalloc_sort_matches_allocating_sort_twice():
    import potreeconverter_b200 as pc
    lib = pc.load_library()
    rng = np.random.default_rng(2024)
    with pc.Context() as ctx:
        # a large call (block-level partitions) and then a small one with
        # many ties (warp-level), reusing the static scratch
        for keys in (rng.random(MAX), rng.integers(0, 9, 3000).astype(np.float64)):
            st, perm = _noalloc_sort(lib, keys)
            assert st == 0
            assert (perm == ctx.sort_keys(keys)).all()


def test_noalloc_sort_rejects_oversize_input():
    import potreeconverter_b200 as pc
    lib = pc.load_library()
    assert lib.pcg_kernel_sort_keys_noalloc(None, MAX + 1, None, None) == 1  # PCG_BAD_INPUT
