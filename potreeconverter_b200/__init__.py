"""B200-native octree LOD builder with PotreeConverter 2.0's output format.

The conversion runs as CUDA kernels for sm_100a inside ``libpcgpu.so``; this
package is a thin ctypes layer over its C ABI (``include/pcgpu.h``), mirroring
the reference's conversion entry (``PotreeConverter <source> ... -o <dir> -m
poisson|poisson_average|random [--attributes ...]``, main.cpp:497-569) as
:func:`convert`: LAS or LAZ file images, one or several converted as one
cloud (:func:`curate_sources` expands paths like the reference).

There is no CPU fallback: importing works without a GPU, but every call that
converts or launches a kernel raises if the CUDA library or a device is
missing.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpcgpu.so")

METHODS = {"poisson": 0, "poisson_average": 1, "random": 2}
RECORDS = {"auto": 0, "resident": 1, "streamed": 2}
FORMS = {"batched": 0, "plain": 1}
PINNED_SEED = 1592614637

STATUS = {0: "ok", 1: "bad input", 2: "point outside bounding box", 3: "out of memory", 4: "timeout",
          5: "internal error", 6: "cuda error", 7: "not found"}


class PcgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS.get(status, status)}: {message}")
        self.status = status


class _Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("random_seed", ctypes.c_uint32), ("form", ctypes.c_int32),
                ("records", ctypes.c_int32), ("stream", ctypes.c_void_p), ("group_points", ctypes.c_int64)]


class _Part(ctypes.Structure):
    _fields_ = [("data", ctypes.POINTER(ctypes.c_uint8)), ("size", ctypes.c_uint64)]


class _Source(ctypes.Structure):
    _fields_ = [("las", ctypes.c_void_p), ("las_size", ctypes.c_uint64), ("device_records", ctypes.c_void_p)]


class _Job(ctypes.Structure):
    _fields_ = [("las", ctypes.c_void_p), ("las_size", ctypes.c_uint64), ("method", ctypes.c_int32),
                ("flags", ctypes.c_int32), ("name", ctypes.c_char_p), ("projection", ctypes.c_char_p),
                ("device_records", ctypes.c_void_p), ("num_sources", ctypes.c_int32),
                ("num_attributes", ctypes.c_int32), ("sources", ctypes.POINTER(_Source)),
                ("attributes", ctypes.POINTER(ctypes.c_char_p))]


OCTREE_ON_DEVICE = 1


@dataclass
class Resident:
    """A source whose point records are already in device memory: `header`
    holds the file's header and VLRs (a LAS or LAZ image, points not
    needed), `device_records` the device address of its decoded records
    (point count x record length bytes)."""
    header: bytes
    device_records: int


class _Stats(ctypes.Structure):
    _fields_ = [("num_points", ctypes.c_int64), ("num_chunks", ctypes.c_int64), ("num_nodes", ctypes.c_int64),
                ("output_points", ctypes.c_int64), ("octree_depth", ctypes.c_int64),
                ("escalated_pairs", ctypes.c_int64), ("heapsort_fallbacks", ctypes.c_int64),
                ("ms_total", ctypes.c_double), ("ms_h2d", ctypes.c_double), ("ms_chunking", ctypes.c_double),
                ("ms_octree", ctypes.c_double), ("ms_sampling", ctypes.c_double), ("ms_output", ctypes.c_double),
                ("ms_d2h", ctypes.c_double), ("ms_host_writers", ctypes.c_double), ("gpu_launches", ctypes.c_int64),
                ("ms_sort", ctypes.c_double), ("ms_greedy", ctypes.c_double), ("sampled_nodes", ctypes.c_int64),
                ("candidates", ctypes.c_int64), ("replayed_nodes", ctypes.c_int64),
                ("replayed_candidates", ctypes.c_int64), ("ms_lists", ctypes.c_double), ("list_entries", ctypes.c_int64),
                ("cluster_nodes", ctypes.c_int64), ("ms_decode", ctypes.c_double), ("laz_chunks", ctypes.c_int64),
                ("device_peak_bytes", ctypes.c_int64), ("parts", ctypes.c_int64), ("survivors", ctypes.c_int64),
                ("records_resident", ctypes.c_int64), ("device_estimate_bytes", ctypes.c_int64)]


class _Node(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char_p), ("num_points", ctypes.c_int64), ("byte_offset", ctypes.c_uint64),
                ("byte_size", ctypes.c_uint64)]


class _Result(ctypes.Structure):
    _fields_ = [("octree", ctypes.POINTER(ctypes.c_uint8)), ("octree_size", ctypes.c_uint64),
                ("hierarchy", ctypes.POINTER(ctypes.c_uint8)), ("hierarchy_size", ctypes.c_uint64),
                ("metadata", ctypes.c_char_p), ("metadata_size", ctypes.c_uint64), ("stats", _Stats),
                ("nodes", ctypes.POINTER(_Node)), ("num_nodes", ctypes.c_uint64),
                ("octree_parts", ctypes.POINTER(_Part)), ("num_octree_parts", ctypes.c_uint64)]


class _Chunk(ctypes.Structure):
    _fields_ = [("id", ctypes.c_char * 16), ("level", ctypes.c_int32), ("x", ctypes.c_int32), ("y", ctypes.c_int32),
                ("z", ctypes.c_int32), ("count", ctypes.c_int64)]


class _OctreeNode(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 32), ("start", ctypes.c_int64), ("count", ctypes.c_int64),
                ("is_leaf", ctypes.c_int32), ("pad", ctypes.c_int32)]


# every symbol include/pcgpu.h declares
EXPORTS = ["pcg_create", "pcg_destroy", "pcg_last_error", "pcg_status_string", "pcg_convert", "pcg_result_free",
           "pcg_write_files", "pcg_submit", "pcg_poll", "pcg_wait", "pcg_kernel_sort_keys", "pcg_kernel_shuffle",
           "pcg_kernel_sort_keys_noalloc", "pcg_kernel_laz_decode", "pcg_kernel_decode_count", "pcg_kernel_lut",
           "pcg_kernel_scatter", "pcg_kernel_octree", "pcg_kernel_accept"]

_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libpcgpu.so (built by ``python -m potreeconverter_b200.build``)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"libpcgpu.so not found at {path}; build it with python -m potreeconverter_b200.build")
    lib = ctypes.CDLL(path)
    c = ctypes
    lib.pcg_create.argtypes = [c.POINTER(c.c_void_p), c.POINTER(_Opts)]
    lib.pcg_destroy.argtypes = [c.c_void_p]
    lib.pcg_last_error.argtypes = [c.c_void_p]
    lib.pcg_last_error.restype = c.c_char_p
    lib.pcg_status_string.argtypes = [c.c_int]
    lib.pcg_status_string.restype = c.c_char_p
    lib.pcg_convert.argtypes = [c.c_void_p, c.POINTER(_Job), c.POINTER(_Result)]
    lib.pcg_result_free.argtypes = [c.POINTER(_Result)]
    lib.pcg_write_files.argtypes = [c.POINTER(_Result), c.c_char_p]
    lib.pcg_submit.argtypes = [c.c_void_p, c.POINTER(_Job), c.POINTER(c.c_uint64)]
    lib.pcg_poll.argtypes = [c.c_void_p, c.c_uint64, c.POINTER(c.c_int32)]
    lib.pcg_wait.argtypes = [c.c_void_p, c.c_uint64, c.POINTER(_Result)]
    lib.pcg_kernel_sort_keys.argtypes = [c.c_void_p, c.c_void_p, c.c_int64, c.c_void_p]
    lib.pcg_kernel_shuffle.argtypes = [c.c_void_p, c.c_int64, c.c_uint32, c.c_void_p]
    lib.pcg_kernel_sort_keys_noalloc.argtypes = [c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p]
    lib.pcg_kernel_laz_decode.argtypes = [c.c_void_p, c.c_char_p, c.c_uint64, c.c_void_p, c.c_uint64]
    lib.pcg_kernel_decode_count.argtypes = [c.c_void_p, c.c_char_p, c.c_uint64, c.c_void_p, c.c_void_p, c.c_void_p,
                                            c.c_void_p, c.c_int64, c.c_void_p, c.c_int64, c.POINTER(c.c_int32)]
    lib.pcg_kernel_lut.argtypes = [c.c_void_p, c.c_void_p, c.c_int32, c.c_int64, c.c_void_p, c.POINTER(_Chunk), c.c_int64,
                                   c.POINTER(c.c_int32)]
    lib.pcg_kernel_scatter.argtypes = [c.c_void_p, c.c_void_p, c.c_int64, c.c_void_p, c.c_int32, c.c_int32, c.c_void_p,
                                       c.c_void_p]
    lib.pcg_kernel_octree.argtypes = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_int64, c.c_void_p, c.c_void_p,
                                      c.c_void_p, c.c_void_p, c.c_char_p, c.c_void_p, c.POINTER(_OctreeNode), c.c_int64,
                                      c.POINTER(c.c_int64), c.POINTER(c.c_int64)]
    lib.pcg_kernel_accept.argtypes = [c.c_void_p, c.c_int32, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p,
                                      c.c_int64, c.c_void_p, c.c_void_p, c.c_void_p, c.c_void_p, c.c_double, c.c_void_p,
                                      c.c_void_p]
    _lib = lib
    return lib


@dataclass
class Conversion:
    """The three PotreeConverter outputs plus run statistics and the nodes
    in completion order as (name, byte offset, byte size, points)."""
    octree: bytes
    hierarchy: bytes
    metadata: str
    stats: dict
    nodes: list

    def write(self, outdir: str) -> None:
        os.makedirs(outdir, exist_ok=True)
        with open(os.path.join(outdir, "octree.bin"), "wb") as f:
            f.write(self.octree)
        with open(os.path.join(outdir, "hierarchy.bin"), "wb") as f:
            f.write(self.hierarchy)
        with open(os.path.join(outdir, "metadata.json"), "w", newline="") as f:
            f.write(self.metadata)


def _copy_out(ptr, size: int) -> bytes:
    """Bytes at a library buffer; ctypes.string_at takes a 32-bit size, so
    images of 2 GiB and more are copied with memmove."""
    if not size:
        return b""
    if not ptr:
        raise ValueError("no buffer behind a non-empty result")
    if size < (1 << 31):
        return ctypes.string_at(ptr, size)
    buf = bytearray(size)
    ctypes.memmove((ctypes.c_char * size).from_buffer(buf), ptr, size)
    return bytes(buf)


def _take(lib, res: _Result) -> Conversion:
    if res.octree or not res.octree_parts:
        octree = _copy_out(res.octree, res.octree_size)
    else:  # a conversion in parts: octree.bin is its pieces back to back
        octree = b"".join(_copy_out(res.octree_parts[i].data, res.octree_parts[i].size)
                          for i in range(res.num_octree_parts))
    hierarchy = _copy_out(res.hierarchy, res.hierarchy_size)
    metadata = ctypes.string_at(res.metadata, res.metadata_size).decode() if res.metadata_size else ""
    stats = {name: getattr(res.stats, name) for name, _ in _Stats._fields_}
    nodes = [(res.nodes[i].name.decode(), res.nodes[i].byte_offset, res.nodes[i].byte_size, res.nodes[i].num_points)
             for i in range(res.num_nodes)] if res.nodes else []
    lib.pcg_result_free(ctypes.byref(res))
    return Conversion(octree, hierarchy, metadata, stats, nodes)


class Context:
    """A device context (pcg_create/pcg_destroy)."""

    def __init__(self, device: int = 0, seed: int = PINNED_SEED, form: str = "batched", stream: int | None = None,
                 group_points: int = 0, records: str = "auto"):
        """group_points > 0 converts one-file jobs of more points in parts
        of at most that many points; records ("auto", "resident",
        "streamed") places the records of such conversions."""
        self._lib = load_library()
        opts = _Opts(device, seed, FORMS[form], RECORDS[records], stream, group_points)
        h = ctypes.c_void_p()
        st = self._lib.pcg_create(ctypes.byref(h), ctypes.byref(opts))
        if st != 0:
            raise PcgError(st, "pcg_create failed")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.pcg_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _err(self, st):
        return PcgError(st, self._lib.pcg_last_error(self._h).decode(errors="replace"))

    @staticmethod
    def _image(las, keep):
        """(pointer, size) of one LAS image: bytes, a writable buffer, or
        (host pointer, size) already."""
        if isinstance(las, bytes):
            # the library only reads the image: pass the bytes object's own buffer
            keep.append(las)
            return ctypes.cast(ctypes.c_char_p(las), ctypes.c_void_p).value, len(las)
        if isinstance(las, (bytearray, memoryview)):
            buf = (ctypes.c_uint8 * len(las)).from_buffer(las)
            keep.append(buf)
            return ctypes.addressof(buf), len(las)
        return las  # (pointer, size), e.g. pinned host memory

    @classmethod
    def _job(cls, las, method, name, projection, keep, device_records=None, flags=0, attributes=None):
        """las: one LAS image, or a list of images converted as one cloud in
        that order (the reference's source list)."""
        nm = name.encode()
        pj = projection.encode()
        keep.extend([nm, pj])
        if isinstance(las, list):
            def source(img):
                if isinstance(img, Resident):
                    return _Source(*cls._image(img.header, keep), img.device_records)
                return _Source(*cls._image(img, keep), None)
            srcs = (_Source * len(las))(*[source(img) for img in las])
            keep.append(srcs)
            job = _Job(None, 0, METHODS[method], flags, nm, pj, None)
            job.num_sources = len(las)
            job.sources = srcs
        else:
            ptr, size = cls._image(las, keep)
            job = _Job(ptr, size, METHODS[method], flags, nm, pj, device_records)
        if attributes:
            names = (ctypes.c_char_p * len(attributes))(*[a.encode() for a in attributes])
            keep.append(names)
            job.num_attributes = len(attributes)
            job.attributes = names
        return job

    def convert(self, las, method: str = "poisson", name: str = "cloud", projection: str = "",
                attributes=None) -> Conversion:
        """Converts one LAS or LAZ file image (bytes, or (host pointer, size)), or a
        list of images as one point cloud. attributes: the --attributes
        list (None keeps every attribute)."""
        keep = []
        job = self._job(las, method, name, projection, keep, attributes=attributes)
        res = _Result()
        st = self._lib.pcg_convert(self._h, ctypes.byref(job), ctypes.byref(res))
        if st != 0:
            raise self._err(st)
        return _take(self._lib, res)

    def write_files(self, las, out_dir: str, method: str = "poisson", name: str = "cloud", attributes=None) -> dict:
        """Converts and writes octree.bin, hierarchy.bin and metadata.json
        into out_dir (pcg_write_files); returns the statistics."""
        keep = []
        job = self._job(las, method, name, "", keep, attributes=attributes)
        res = _Result()
        st = self._lib.pcg_convert(self._h, ctypes.byref(job), ctypes.byref(res))
        if st != 0:
            raise self._err(st)
        try:
            st = self._lib.pcg_write_files(ctypes.byref(res), out_dir.encode())
            if st != 0:
                raise PcgError(st, f"cannot write into {out_dir}")
            return {n: getattr(res.stats, n) for n, _ in _Stats._fields_}
        finally:
            self._lib.pcg_result_free(ctypes.byref(res))

    def convert_stats(self, las, method: str = "poisson", name: str = "cloud", attributes=None) -> dict:
        """Converts like :meth:`convert` (octree.bin lands in pinned host
        memory) but returns only the statistics, releasing the outputs."""
        keep = []
        job = self._job(las, method, name, "", keep, attributes=attributes)
        res = _Result()
        st = self._lib.pcg_convert(self._h, ctypes.byref(job), ctypes.byref(res))
        if st != 0:
            raise self._err(st)
        stats = {n: getattr(res.stats, n) for n, _ in _Stats._fields_}
        stats["octree_size"] = res.octree_size
        self._lib.pcg_result_free(ctypes.byref(res))
        return stats

    def convert_resident(self, header, device_records: int, method: str = "poisson", name: str = "cloud") -> dict:
        """Converts point records already in device memory; octree.bin stays
        on the device and is released at once. Returns the run statistics."""
        keep = []
        job = self._job(header, method, name, "", keep, device_records=device_records, flags=OCTREE_ON_DEVICE)
        res = _Result()
        st = self._lib.pcg_convert(self._h, ctypes.byref(job), ctypes.byref(res))
        if st != 0:
            raise self._err(st)
        stats = {n: getattr(res.stats, n) for n, _ in _Stats._fields_}
        stats["octree_size"] = res.octree_size
        self._lib.pcg_result_free(ctypes.byref(res))
        return stats

    def submit(self, las, method: str = "poisson", name: str = "cloud", projection: str = "", attributes=None) -> int:
        """Queues a conversion (the images are copied at once); returns its id."""
        keep = []
        job = self._job(las, method, name, projection, keep, attributes=attributes)
        jid = ctypes.c_uint64()
        st = self._lib.pcg_submit(self._h, ctypes.byref(job), ctypes.byref(jid))
        if st != 0:
            raise self._err(st)
        return jid.value

    def poll(self, job_id: int) -> bool:
        done = ctypes.c_int32()
        st = self._lib.pcg_poll(self._h, job_id, ctypes.byref(done))
        if st != 0:
            raise self._err(st)
        return bool(done.value)

    def wait(self, job_id: int) -> Conversion:
        res = _Result()
        st = self._lib.pcg_wait(self._h, job_id, ctypes.byref(res))
        if st != 0:
            raise self._err(st)
        return _take(self._lib, res)

    def sort_keys(self, keys):
        """Permutation std::sort produces for FP64 keys (device kernel)."""
        import numpy as np
        k = np.ascontiguousarray(keys, dtype=np.float64)
        perm = np.empty(k.shape[0], dtype=np.int32)
        st = self._lib.pcg_kernel_sort_keys(self._h, k.ctypes.data, k.shape[0], perm.ctypes.data)
        if st != 0:
            raise self._err(st)
        return perm

    def decode_count(self, las: bytes):
        """The counting pass on the device: (X, Y, Z, cell, grid) as numpy
        arrays (the grid flattened, G^3 counts)."""
        import struct
        import numpy as np
        hdr = struct.unpack_from("<H", las, 94)[0]
        n = struct.unpack_from("<I", las, 107)[0]
        if las[25] >= 4 and hdr >= 375:
            n = max(n, struct.unpack_from("<Q", las, 247)[0])
        g = 128 if n < 100_000_000 else (256 if n < 500_000_000 else 512)
        X, Y, Z = (np.empty(max(n, 1), np.int32) for _ in range(3))
        cell = np.empty(max(n, 1), np.uint32)
        grid = np.empty(g ** 3, np.uint32)
        gs = ctypes.c_int32()
        st = self._lib.pcg_kernel_decode_count(self._h, ctypes.c_char_p(las), len(las), X.ctypes.data, Y.ctypes.data,
                                               Z.ctypes.data, cell.ctypes.data, X.size, grid.ctypes.data, grid.size,
                                               ctypes.byref(gs))
        if st != 0:
            raise self._err(st)
        return X[:n], Y[:n], Z[:n], cell[:n], grid[: gs.value ** 3]

    def lut(self, grid, grid_size: int, max_points_per_chunk: int):
        """The chunker's LUT merge of a count grid (G^3 counts): (chunks, lut)
        with chunks a list of (id, level, x, y, z, count) in chunk file-name
        order and lut every cell's index in that list (-1: no chunk)."""
        import numpy as np
        g = np.ascontiguousarray(grid, dtype=np.uint32)
        lut = np.empty(grid_size ** 3, np.int32)
        cap = 1 << 16
        while True:
            chunks = (_Chunk * cap)()
            num = ctypes.c_int32()
            st = self._lib.pcg_kernel_lut(self._h, g.ctypes.data, grid_size, max_points_per_chunk, lut.ctypes.data, chunks, cap,
                                          ctypes.byref(num))
            if st == 1 and num.value > cap:
                cap = num.value
                continue
            if st != 0:
                raise self._err(st)
            out = [(c.id.decode(), c.level, c.x, c.y, c.z, c.count) for c in chunks[: num.value]]
            return out, lut

    def scatter(self, cell, lut, grid_size: int, num_chunks: int):
        """Points distributed to chunks: (ids, chunk_start), ids grouped by
        chunk in input order, chunk_start num_chunks + 1 offsets."""
        import numpy as np
        c = np.ascontiguousarray(cell, dtype=np.uint32)
        lt = np.ascontiguousarray(lut, dtype=np.int32)
        ids = np.empty(max(c.shape[0], 1), np.uint32)
        start = np.empty(num_chunks + 1, np.int64)
        st = self._lib.pcg_kernel_scatter(self._h, c.ctypes.data, c.shape[0], lt.ctypes.data, grid_size, num_chunks,
                                          ids.ctypes.data, start.ctypes.data)
        if st != 0:
            raise self._err(st)
        return ids[: c.shape[0]], start

    def octree(self, X, Y, Z, scale, offset, box_min, box_max, root_name: str = "r"):
        """One chunk's octree: (order, nodes, depth); nodes a list of
        (name, start, count, is_leaf) sorted by name, order the points'
        indices in the order the octree build leaves them."""
        import numpy as np
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (X, Y, Z)]
        vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in (scale, offset, box_min, box_max)]
        n = arrs[0].shape[0]
        order = np.empty(max(n, 1), np.uint32)
        cap = 4096
        while True:
            nodes = (_OctreeNode * cap)()
            num, depth = ctypes.c_int64(), ctypes.c_int64()
            st = self._lib.pcg_kernel_octree(self._h, *[a.ctypes.data for a in arrs], n, *[v.ctypes.data for v in vecs],
                                             root_name.encode(), order.ctypes.data, nodes, cap, ctypes.byref(num),
                                             ctypes.byref(depth))
            if st == 1 and num.value > cap:
                cap = num.value
                continue
            if st != 0:
                raise self._err(st)
            out = [(x.name.decode(), x.start, x.count, x.is_leaf) for x in nodes[: num.value]]
            return order[:n], out, depth.value

    def accept(self, method: str, X, Y, Z, child, scale, offset, box_min, box_max, spacing: float, rgb=None):
        """One inner node's sampler decision: (accepted, rgb) with accepted
        a 0/1 mask over the candidates (children's points in order) and rgb
        the averaged colours (poisson_average) or None."""
        import numpy as np
        arrs = [np.ascontiguousarray(a, dtype=np.int32) for a in (X, Y, Z)]
        ch = np.ascontiguousarray(child, dtype=np.uint8)
        vecs = [np.ascontiguousarray(v, dtype=np.float64) for v in (scale, offset, box_min, box_max)]
        n = ch.shape[0]
        acc = np.empty(max(n, 1), np.uint8)
        col_in = np.ascontiguousarray(rgb, dtype=np.uint16) if rgb is not None else None
        col_out = np.empty((max(n, 1), 3), np.uint16) if method == "poisson_average" else None
        st = self._lib.pcg_kernel_accept(self._h, METHODS[method], *[a.ctypes.data for a in arrs], ch.ctypes.data,
                                         col_in.ctypes.data if col_in is not None else None, n,
                                         *[v.ctypes.data for v in vecs], spacing, acc.ctypes.data,
                                         col_out.ctypes.data if col_out is not None else None)
        if st != 0:
            raise self._err(st)
        return acc[:n], (col_out[:n] if col_out is not None else None)

    def laz_decode(self, laz: bytes) -> bytes:
        """Point records of a LAZ file image, decoded on the device."""
        import struct
        hdr = struct.unpack_from("<H", laz, 94)[0]
        n = struct.unpack_from("<I", laz, 107)[0]
        if laz[25] >= 4 and hdr >= 375:
            n = max(n, struct.unpack_from("<Q", laz, 247)[0])
        size = n * struct.unpack_from("<H", laz, 105)[0]
        out = ctypes.create_string_buffer(max(1, size))
        st = self._lib.pcg_kernel_laz_decode(self._h, ctypes.c_char_p(laz), len(laz), out, size)
        if st != 0:
            raise self._err(st)
        return out.raw[:size]

    def shuffle(self, n: int, seed: int = PINNED_SEED):
        """Index order std::shuffle(iota(n), default_random_engine(seed)) gives (device kernel)."""
        import numpy as np
        perm = np.empty(n, dtype=np.int32)
        st = self._lib.pcg_kernel_shuffle(self._h, n, seed, perm.ctypes.data)
        if st != 0:
            raise self._err(st)
        return perm


def convert(las, method: str = "poisson", name: str = "cloud", form: str = "batched", seed: int = PINNED_SEED,
            device: int = 0, attributes=None) -> Conversion:
    """One-shot conversion: PotreeConverter <in.las> [<in.las> ...] -m method
    [--attributes ...]; las is one image or a list of images."""
    with Context(device=device, seed=seed, form=form) as ctx:
        return ctx.convert(las, method=method, name=name, attributes=attributes)


def curate_sources(paths) -> tuple:
    """The reference's input list (curateSources, main.cpp:146-200): every
    path that is a directory contributes its entries whose names end in
    "las" or "laz" (case-insensitive), in name order (the pinned order);
    files are taken when their names end so. Returns (name, paths), name
    being the stem of the first path given."""
    expanded = []
    name = ""
    for p in paths:
        if os.path.isdir(p):
            for e in sorted(os.listdir(p)):
                full = os.path.join(p, e)
                if e.lower().endswith(("las", "laz")):
                    expanded.append(full)
        elif os.path.isfile(p) and p.lower().endswith(("las", "laz")):
            expanded.append(p)
        if not name:
            name = os.path.splitext(os.path.basename(p))[0]  # fs::path(p).stem()
    return name, expanded
