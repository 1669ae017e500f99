"""The Python binding copies library buffers of any size (ctypes.string_at
alone stops at 2 GiB)."""

import ctypes

from potreeconverter_b200 import _copy_out


def test_copy_out_small_and_empty():
    src = (ctypes.c_uint8 * 5)(1, 2, 3, 4, 5)
    assert _copy_out(ctypes.addressof(src), 5) == bytes([1, 2, 3, 4, 5])
    assert _copy_out(None, 0) == b""
