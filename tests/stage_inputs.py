"""Inputs of the stage-level parity tests, derived from a synthetic LAS image
through the oracle: the counting pass, the chunk list, the distribution to
chunks, one chunk's points with its cube, and inner nodes' candidates. Both
the library's stage entry points and the oracle's stage hooks are then fed
the same arrays. Test infrastructure only."""

from __future__ import annotations

import struct

import numpy as np


def header_transform(las: bytes):
    """(scale, offset, cube_min, cube_size) of the conversion of one LAS
    file: offset = header min; scale = max(header scale, extent / 2^30)
    (computeScaleOffset, PotreeConverter.h:29-76); the cube spans the
    largest extent from the header min (main.cpp:237-239)."""
    scale = np.array(struct.unpack_from("<3d", las, 131))
    mx = np.array(struct.unpack_from("<6d", las, 179)[0::2])
    mn = np.array(struct.unpack_from("<6d", las, 179)[1::2])
    ext = mx - mn
    out_scale = np.array([max(scale.min(), e / 2 ** 30) for e in ext])
    return out_scale, mn.copy(), mn.copy(), float(ext.max())


def node_box(cube_min, cube_size: float, name: str):
    """The box of an octree node named "r" + octant digits (childBoundingBoxOf,
    converter_utils.h:106-136; bit 2 = x, bit 1 = y, bit 0 = z)."""
    bmin = np.array(cube_min, dtype=np.float64)
    bmax = bmin + cube_size
    for ch in name[1:]:
        i = int(ch)
        size = bmax - bmin
        ctr = bmin + size * 0.5
        for a, bit in ((0, 4), (1, 2), (2, 1)):
            if i & bit:
                bmin[a] = ctr[a]
            else:
                bmax[a] = ctr[a]
    return bmin, bmax


def max_points_per_chunk(n: int) -> int:
    return min(n // 20, 10_000_000)  # chunker_countsort_laszip.cpp:1210-1211


class StageInputs:
    def __init__(self, oracle, las: bytes):
        self.las = las
        self.X, self.Y, self.Z, self.cell, self.grid = oracle.decode_count(las)
        self.n = self.X.shape[0]
        self.G = int(round(self.grid.shape[0] ** (1 / 3)))
        self.mpc = max_points_per_chunk(self.n)
        self.scale, self.offset, self.cube_min, self.cube_size = header_transform(las)
        self.chunks, self.lut = oracle.lut(self.grid, self.G, self.mpc)
        self.ids, self.chunk_start = oracle.scatter(self.cell, self.lut, len(self.chunks))

    def chunk_points(self, k: int):
        """Chunk k's points in chunk order (X, Y, Z) with its id and cube."""
        sel = self.ids[self.chunk_start[k]: self.chunk_start[k + 1]]
        name = self.chunks[k][0]
        bmin, bmax = node_box(self.cube_min, self.cube_size, name)
        return self.X[sel], self.Y[sel], self.Z[sel], name, bmin, bmax

    def largest_chunks(self, count: int):
        sizes = np.diff(self.chunk_start)
        return [int(k) for k in np.argsort(-sizes, kind="stable")[:count]]

    def node_candidates(self, X, Y, Z, name: str):
        """Points of a node as the candidates its sampler sees when its
        children are leaves holding them: grouped by child octant (child 0
        first), input order inside a child. Returns (X, Y, Z, child, box
        min, box max, spacing)."""
        bmin, bmax = node_box(self.cube_min, self.cube_size, name)
        ctr = bmin + (bmax - bmin) * 0.5
        x = X * self.scale[0] + self.offset[0]
        y = Y * self.scale[1] + self.offset[1]
        z = Z * self.scale[2] + self.offset[2]
        child = ((x >= ctr[0]).astype(np.uint8) << 2) | ((y >= ctr[1]).astype(np.uint8) << 1) | (z >= ctr[2]).astype(np.uint8)
        order = np.argsort(child, kind="stable")
        level = len(name) - 1
        spacing = (self.cube_size / 128.0) / 2.0 ** level
        return X[order], Y[order], Z[order], child[order], bmin, bmax, spacing
