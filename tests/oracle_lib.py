"""Test-side access to the oracle (oracle/pcref.cpp, the single-threaded
CPU restatement of the reference pipeline) and to the golden fixtures the
pinned reference produced (tests/golden/golden.json). Test infrastructure
only: nothing in the library imports this module."""

from __future__ import annotations

import ctypes
import functools
import hashlib
import json
import os
import subprocess

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "libpcref.so")
GOLDEN = os.path.join(REPO, "tests", "golden", "golden.json")
PINNED_SEED = 1592614637


class _Out(ctypes.Structure):
    _fields_ = [("octree", ctypes.POINTER(ctypes.c_uint8)), ("octree_size", ctypes.c_uint64),
                ("hierarchy", ctypes.POINTER(ctypes.c_uint8)), ("hierarchy_size", ctypes.c_uint64),
                ("metadata", ctypes.c_char_p), ("metadata_size", ctypes.c_uint64),
                ("num_chunks", ctypes.c_int32), ("chunk_ids", ctypes.c_void_p),
                ("chunk_counts", ctypes.POINTER(ctypes.c_int64)), ("error", ctypes.c_char * 256),
                ("num_nodes", ctypes.c_int64), ("node_names", ctypes.c_void_p), ("node_info", ctypes.POINTER(ctypes.c_int64))]


def build_oracle():
    if not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "restatement"], check=True)


class Oracle:
    def __init__(self):
        build_oracle()
        lib = ctypes.CDLL(ORACLE_LIB)
        lib.pcref_convert.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_char_p,
                                      ctypes.c_uint32, ctypes.POINTER(_Out)]
        lib.pcref_convert_sources.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                              ctypes.c_int32, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32,
                                              ctypes.POINTER(_Out)]
        lib.pcref_free.argtypes = [ctypes.POINTER(_Out)]
        lib.pcref_decode_count.argtypes = [ctypes.c_void_p, ctypes.c_uint64] + [ctypes.c_void_p] * 5 + [
            ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_char_p]
        lib.pcref_std_sort_perm.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
        lib.pcref_lut.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
        lib.pcref_scatter.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p,
                                      ctypes.c_void_p]
        lib.pcref_octree.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] + [ctypes.c_void_p] * 4 + [
            ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
            ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        lib.pcref_accept.argtypes = [ctypes.c_int32] + [ctypes.c_void_p] * 5 + [ctypes.c_int64] + [ctypes.c_void_p] * 4 + [
            ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        lib.pcref_std_shuffle.argtypes = [ctypes.c_int64, ctypes.c_uint32, ctypes.c_void_p]
        self.lib = lib

    def convert(self, las: bytes, method: str, name: str = "cloud", seed: int = PINNED_SEED):
        return self.convert_sources([las], method, name=name, seed=seed)

    def convert_sources(self, sources, method: str, name: str = "cloud", seed: int = PINNED_SEED, attributes=()):
        """Several LAS images as one cloud, in order, keeping only
        `attributes` when given (the reference's --attributes)."""
        bufs = [(ctypes.c_uint8 * len(las)).from_buffer_copy(las) for las in sources]
        ptrs = (ctypes.c_void_p * len(bufs))(*[ctypes.addressof(b) for b in bufs])
        sizes = (ctypes.c_uint64 * len(bufs))(*[len(las) for las in sources])
        names = [a.encode() for a in attributes]
        arr = (ctypes.c_char_p * max(1, len(names)))(*names)
        out = _Out()
        rc = self.lib.pcref_convert_sources(ptrs, sizes, len(bufs), arr, len(names), method.encode(), name.encode(),
                                            seed, ctypes.byref(out))
        if rc != 0:
            raise RuntimeError(out.error.decode())
        res = {
            "octree.bin": ctypes.string_at(out.octree, out.octree_size),
            "hierarchy.bin": ctypes.string_at(out.hierarchy, out.hierarchy_size),
            "metadata.json": ctypes.string_at(out.metadata, out.metadata_size),
        }
        p = out.chunk_ids
        chunk_ids = []
        off = 0
        for _ in range(out.num_chunks):
            s = ctypes.string_at(p + off)
            chunk_ids.append(s.decode())
            off += len(s) + 1
        res["chunks"] = list(zip(chunk_ids, [out.chunk_counts[i] for i in range(out.num_chunks)]))
        nodes = []
        off = 0
        for i in range(out.num_nodes):
            s = ctypes.string_at(out.node_names + off)
            off += len(s) + 1
            nodes.append((s.decode(), out.node_info[3 * i], out.node_info[3 * i + 1], out.node_info[3 * i + 2]))
        res["nodes"] = nodes  # completion order: (name, byte offset, byte size, points)
        self.lib.pcref_free(ctypes.byref(out))
        return res

    def decode_count(self, las: bytes):
        """The counting pass (countPointsInCells): X, Y, Z, cell, grid."""
        import struct
        hdr = struct.unpack_from("<H", las, 94)[0]
        n = struct.unpack_from("<I", las, 107)[0]
        if las[25] >= 4 and hdr >= 375:
            n = max(n, struct.unpack_from("<Q", las, 247)[0])
        buf = (ctypes.c_uint8 * len(las)).from_buffer_copy(las)
        X, Y, Z = (np.empty(max(n, 1), np.int32) for _ in range(3))
        cell = np.empty(max(n, 1), np.uint32)
        grid = np.empty(512 ** 3 if n >= 100_000_000 else 128 ** 3, np.int64)
        gs = ctypes.c_int64()
        err = ctypes.create_string_buffer(256)
        rc = self.lib.pcref_decode_count(ctypes.addressof(buf), len(las), X.ctypes.data, Y.ctypes.data, Z.ctypes.data,
                                         cell.ctypes.data, grid.ctypes.data, grid.size, ctypes.byref(gs), err)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return X[:n], Y[:n], Z[:n], cell[:n], grid[: gs.value ** 3]

    def lut(self, grid, grid_size: int, max_points_per_chunk: int):
        """createLUT of a count grid: (chunks, lut) like Context.lut."""
        g = np.ascontiguousarray(grid, dtype=np.int64)
        lut = np.empty(grid_size ** 3, np.int32)
        cap = grid_size ** 3  # at most one chunk per cell
        ids = ctypes.create_string_buffer(16 * cap)
        info = np.empty(5 * cap, np.int64)
        num = ctypes.c_int64()
        if self.lib.pcref_lut(g.ctypes.data, grid_size, max_points_per_chunk, lut.ctypes.data, ids, info.ctypes.data, cap,
                              ctypes.byref(num)) != 0:
            raise RuntimeError("too many chunks")
        out = []
        raw = ids.raw  # one copy of the buffer, not one per chunk
        for k in range(num.value):
            name = raw[16 * k: 16 * k + 16].split(b"\0")[0].decode()
            out.append((name,) + tuple(int(v) for v in info[5 * k: 5 * k + 5]))
        return out, lut

    def scatter(self, cell, lut, num_chunks: int):
        c = np.ascontiguousarray(cell, dtype=np.uint32)
        lt = np.ascontiguousarray(lut, dtype=np.int32)
        ids = np.empty(max(c.shape[0], 1), np.uint32)
        start = np.empty(num_chunks + 1, np.int64)
        if self.lib.pcref_scatter(c.ctypes.data, c.shape[0], lt.ctypes.data, num_chunks, ids.ctypes.data,
                                  start.ctypes.data) != 0:
            raise RuntimeError("cell without chunk")
        return ids[: c.shape[0]], start

    def octree(self, X, Y, Z, scale, offset, box_min, box_max, root_name: str = "r"):
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (X, Y, Z)]
        vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in (scale, offset, box_min, box_max)]
        n = arrs[0].shape[0]
        order = np.empty(max(n, 1), np.uint32)
        cap = 1 << 16
        names = ctypes.create_string_buffer(32 * cap)
        info = np.empty(3 * cap, np.int64)
        num, depth = ctypes.c_int64(), ctypes.c_int64()
        if self.lib.pcref_octree(*[a.ctypes.data for a in arrs], n, *[v.ctypes.data for v in vecs], root_name.encode(),
                                 order.ctypes.data, names, info.ctypes.data, cap, ctypes.byref(num), ctypes.byref(depth)) != 0:
            raise RuntimeError("too many nodes")
        nodes = []
        raw = names.raw
        for k in range(num.value):
            nm = raw[32 * k: 32 * k + 32].split(b"\0")[0].decode()
            nodes.append((nm, int(info[3 * k]), int(info[3 * k + 1]), int(info[3 * k + 2])))
        return order[:n], nodes, depth.value

    def accept(self, method: str, X, Y, Z, child, scale, offset, box_min, box_max, spacing: float, rgb=None):
        m = {"poisson": 0, "poisson_average": 1, "random": 2}[method]
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (X, Y, Z)]
        ch = np.ascontiguousarray(child, dtype=np.uint8)
        vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in (scale, offset, box_min, box_max)]
        n = ch.shape[0]
        acc = np.empty(max(n, 1), np.uint8)
        col_in = np.ascontiguousarray(rgb, dtype=np.uint16) if rgb is not None else None
        col_out = np.empty((max(n, 1), 3), np.uint16) if m == 1 else None
        if self.lib.pcref_accept(m, *[a.ctypes.data for a in arrs], ch.ctypes.data,
                                 col_in.ctypes.data if col_in is not None else None, n, *[v.ctypes.data for v in vecs],
                                 spacing, acc.ctypes.data, col_out.ctypes.data if col_out is not None else None) != 0:
            raise RuntimeError("children not in order")
        return acc[:n], (col_out[:n] if col_out is not None else None)

    def sort_perm(self, keys):
        k = np.ascontiguousarray(keys, dtype=np.float64)
        perm = np.empty(k.shape[0], dtype=np.int32)
        self.lib.pcref_std_sort_perm(k.ctypes.data, k.shape[0], perm.ctypes.data)
        return perm

    def shuffle(self, n, seed=PINNED_SEED):
        perm = np.empty(n, dtype=np.int32)
        self.lib.pcref_std_shuffle(n, seed, perm.ctypes.data)
        return perm


def load_golden():
    with open(GOLDEN) as f:
        return json.load(f)


@functools.lru_cache(maxsize=16)
def case_las(kind: str, n: int, seed: int, kwargs_json: str) -> bytes:
    from potreeconverter_b200 import synth
    return synth.generate(kind, n, seed, **json.loads(kwargs_json))


def las_for(case: dict) -> bytes:
    las = case_las(case["kind"], case["points"], case["seed"], json.dumps(case["kwargs"], sort_keys=True))
    assert hashlib.md5(las).hexdigest() == case["las_md5"], "synthetic generator output changed"
    return las


def md5(b: bytes) -> str:
    return hashlib.md5(b).hexdigest()


@functools.lru_cache(maxsize=8)
def _case_sources(kind: str, n: int, seed: int, kwargs_json: str, order: tuple) -> tuple:
    from potreeconverter_b200 import synth
    imgs = synth.sources(kind, n, seed, **json.loads(kwargs_json))
    return tuple(imgs[k] for k in order)


def sources_for(case: dict) -> list:
    """File images of a multi-source golden case, in the order passed."""
    imgs = _case_sources(case["kind"], case["points"], case["seed"], json.dumps(case["kwargs"], sort_keys=True),
                         tuple(case["order"]))
    assert [hashlib.md5(b).hexdigest() for b in imgs] == case["las_md5"], "synthetic generator output changed"
    return list(imgs)


LAZ_TOOL = os.path.join(ORACLE_DIR, "_ref", "laz_tool")


def have_laz_tool() -> bool:
    return os.path.exists(LAZ_TOOL)


def to_laz(las: bytes, chunk_size: int = 0) -> bytes:
    """The LAZ image the reference's vendored LASzip writes for a LAS image
    (oracle/_ref/laz_tool; chunk_size 0 is LASzip's default)."""
    import tempfile
    with tempfile.TemporaryDirectory() as tmp:
        src, dst = os.path.join(tmp, "in.las"), os.path.join(tmp, "out.laz")
        with open(src, "wb") as f:
            f.write(las)
        subprocess.run([LAZ_TOOL, "compress", src, dst] + ([str(chunk_size)] if chunk_size else []), check=True,
                       capture_output=True)
        with open(dst, "rb") as f:
            return f.read()


def laz_sources_for(case: dict) -> list:
    """Sources of a golden case as the pinned reference was given them: the
    positions the case's "laz" entry lists as LAZ images."""
    imgs = sources_for(case)
    spec = case.get("laz")
    if not spec:
        return imgs
    out, k = [], 0
    for pos, img in enumerate(imgs):
        if pos in spec["sources"]:
            z = to_laz(img, spec["chunk_size"])
            assert hashlib.md5(z).hexdigest() == spec["laz_md5"][k], "LASzip output changed"
            k += 1
            out.append(z)
        else:
            out.append(img)
    return out


def las_records(las: bytes) -> bytes:
    import struct
    return las[struct.unpack_from("<I", las, 96)[0]:]
