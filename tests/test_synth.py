"""Seeded synthetic LAS inputs: deterministic, header box equal to the exact
min/max of the quantized coordinates (the reference exits on points outside
the header box)."""

import struct

import numpy as np
import pytest

from potreeconverter_b200 import synth


@pytest.mark.parametrize("kind", ["terrain", "hotspots", "lattice", "strips", "duplicates", "cube"])
def test_header_box_is_exact(kind):
    las = synth.generate(kind, 20000, 11)
    assert las == synth.generate(kind, 20000, 11)
    off = struct.unpack_from("<I", las, 96)[0]
    rec = struct.unpack_from("<H", las, 105)[0]
    n = struct.unpack_from("<I", las, 107)[0]
    assert n == 20000
    xyz = np.frombuffer(las, dtype=np.uint8, offset=off, count=n * rec).reshape(n, rec)[:, :12].copy().view("<i4")
    mx, mnx, my, mny, mz, mnz = struct.unpack_from("<6d", las, 179)
    assert mnx == xyz[:, 0].min() * 0.001 and mx == xyz[:, 0].max() * 0.001
    assert mny == xyz[:, 1].min() * 0.001 and my == xyz[:, 1].max() * 0.001
    assert mnz == xyz[:, 2].min() * 0.001 and mz == xyz[:, 2].max() * 0.001


@pytest.mark.parametrize("kind,kw", [("strips", {}), ("terrain", {"pdrf": 2}), ("terrain", {"pdrf": 3, "extent": 1500.0})])
def test_gpu_generator_images_are_valid_las(oracle, kind, kw):
    # the torch generator of the large workloads, run on the CPU here: the
    # image parses, every point lies in its header box, and the oracle
    # converts it
    import torch
    from potreeconverter_b200 import synth_gpu
    n = 60_000
    host = torch.empty(400 + n * 34, dtype=torch.uint8)
    img = getattr(synth_gpu, kind)(n, 5, device="cpu", host=host, **kw)
    las = bytes(img.numpy())
    X, Y, Z, cell, grid = oracle.decode_count(las)
    assert X.shape[0] == n and int(grid.sum()) == n
    assert len(oracle.convert(las, "poisson")["octree.bin"]) > 0
