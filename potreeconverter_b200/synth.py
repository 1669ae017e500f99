"""Seeded synthetic LAS generator for the benchmark and parity workloads.

The reference's published numbers use real scans that are not available
here, so every workload is a seeded synthetic cloud with the shapes, sizes
and value distributions of the named configurations:

* ``terrain``  -- 2.5D ground: x, y ~ U[0, extent]; z = three seeded sinusoids
  (amplitudes 2-10 m) + N(0, 0.05 m); 10 % of the points on vertical facades
  5-30 m tall. LAS 1.2, point format 2. RGB is a height ramp +/- 2000.
* ``hotspots`` -- LAS 1.4, point format 3 (GPS time, monotone with 1e-5 s
  jitter) plus one float32 extra-bytes attribute ~ N(0, 1); a 2 x 2 km x 50 m
  slab with 20 Gaussian hot-spots (sigma 5-40 m) at 100x background density.
* ``lattice``  -- precision stress: a jittered cubic lattice whose pitch is
  the level-3 node spacing (cube / 1024), every coordinate moved by +/-1-3
  quantization units. Point format 2.
* ``strips``   -- aerial strips: overlapping 300 m flight strips over a seeded
  value-noise heightfield, 15 % canopy points; point format 3.

All coordinates are quantized to scale 0.001, and the header bounding box is
the exact min/max of the quantized coordinates (the reference rejects points
outside the header box, chunker_countsort_laszip.cpp:236-251).
"""

from __future__ import annotations

import struct

import numpy as np

SCALE = 0.001

# LAS point record dtypes (little endian, packed)
_PDRF2 = np.dtype([
    ("X", "<i4"), ("Y", "<i4"), ("Z", "<i4"), ("intensity", "<u2"),
    ("bits", "u1"), ("classification", "u1"), ("scan_angle_rank", "i1"),
    ("user_data", "u1"), ("point_source_id", "<u2"),
    ("red", "<u2"), ("green", "<u2"), ("blue", "<u2"),
])
_PDRF3 = np.dtype([
    ("X", "<i4"), ("Y", "<i4"), ("Z", "<i4"), ("intensity", "<u2"),
    ("bits", "u1"), ("classification", "u1"), ("scan_angle_rank", "i1"),
    ("user_data", "u1"), ("point_source_id", "<u2"), ("gps_time", "<f8"),
    ("red", "<u2"), ("green", "<u2"), ("blue", "<u2"),
])
_PDRF0 = np.dtype([(n, _PDRF2.fields[n][0]) for n in _PDRF2.names[:9]])
_PDRF1 = np.dtype([(n, _PDRF3.fields[n][0]) for n in _PDRF3.names[:10]])
assert _PDRF0.itemsize == 20 and _PDRF1.itemsize == 28 and _PDRF2.itemsize == 26 and _PDRF3.itemsize == 34
_PDRF = {0: _PDRF0, 1: _PDRF1, 2: _PDRF2, 3: _PDRF3}

# LAS extra-bytes data types (type id of the descriptor) for scalar numpy types
_EXTRA_TYPE_ID = {"u1": 1, "i1": 2, "<u2": 3, "<i2": 4, "<u4": 5, "<i4": 6, "<u8": 7, "<i8": 8, "<f4": 9, "<f8": 10}


def _record_dtype(pdrf: int, extra_float: bool, extras=()) -> np.dtype:
    base = _PDRF[pdrf]
    fields = [(n, base.fields[n][0]) for n in base.names]
    if extra_float:
        fields.append(("extra", "<f4"))
    for e in extras:
        shape = e["values"].shape[1:]
        fields.append((e["name"], e["dtype"], shape) if shape else (e["name"], e["dtype"]))
    return np.dtype(fields)


def _extra_descriptor(name: str, type_id: int, description: str, scale=None, offset=None) -> bytes:
    """One 192-byte extra-bytes descriptor (LAS 1.4 R15 table 24)."""
    rec = bytearray(192)
    rec[2] = type_id
    options = (0b01000 if scale is not None else 0) | (0b10000 if offset is not None else 0)
    rec[3] = options
    nb = name.encode()[:31]
    rec[4:4 + len(nb)] = nb
    if scale is not None:
        struct.pack_into("<3d", rec, 112, *scale)
    if offset is not None:
        struct.pack_into("<3d", rec, 136, *offset)
    db = description.encode()[:31]
    rec[160:160 + len(db)] = db
    return bytes(rec)


def _extra_bytes_vlr(name: str = "extra", description: str = "N(0,1) float", descriptors: bytes | None = None) -> bytes:
    """The extra-bytes VLR (record id 4): by default one float32 descriptor."""
    body = descriptors if descriptors is not None else _extra_descriptor(name, 9, description)
    hdr = bytearray(54)
    hdr[2:2 + 9] = b"LASF_Spec"
    struct.pack_into("<HH", hdr, 18, 4, len(body))
    d = b"Extra bytes"
    hdr[22:22 + len(d)] = d
    return bytes(hdr) + body


def write_las(X, Y, Z, attrs: dict, *, pdrf: int, version_minor: int,
              extra=None, scale=None, offset=None, extras=()) -> bytes:
    """Serialize quantized points into an uncompressed LAS file image.

    ``extra`` is the float32 attribute named "extra"; ``extras`` lists more
    extra-bytes attributes as dicts with ``name``, ``dtype`` (a scalar numpy
    type string of ``_EXTRA_TYPE_ID``), ``values`` of shape (n,) or (n, k)
    for k = 2, 3 elements and an optional ``description``. ``scale`` and
    ``offset`` default to 0.001 and 0."""
    n = int(X.shape[0])
    sc = tuple(scale) if scale is not None else (SCALE, SCALE, SCALE)
    of = tuple(offset) if offset is not None else (0.0, 0.0, 0.0)
    dt = _record_dtype(pdrf, extra is not None, extras)
    recs = np.zeros(n, dtype=dt)
    recs["X"], recs["Y"], recs["Z"] = X, Y, Z
    for k, v in attrs.items():
        if k in dt.names:
            recs[k] = v
    if extra is not None:
        recs["extra"] = extra
    for e in extras:
        recs[e["name"]] = e["values"]
    if extras:
        descs = b"" if extra is None else _extra_descriptor("extra", 9, "N(0,1) float")
        for e in extras:
            k = e["values"].shape[1] if e["values"].ndim > 1 else 1
            tid = _EXTRA_TYPE_ID[e["dtype"]] + 10 * (k - 1)
            descs += _extra_descriptor(e["name"], tid, e.get("description", ""))
        vlrs = _extra_bytes_vlr(descriptors=descs)
    else:
        vlrs = _extra_bytes_vlr() if extra is not None else b""

    # LASzip's coordinate: scale * X + offset (the header box holds them all)
    xs = X.astype(np.float64) * sc[0] + of[0]
    ys = Y.astype(np.float64) * sc[1] + of[1]
    zs = Z.astype(np.float64) * sc[2] + of[2]
    ret = (recs["bits"] & 7).astype(np.int64)
    byret = np.bincount(np.clip(ret, 1, 5) - 1, minlength=5)[:5] if n else np.zeros(5, np.int64)
    bbox = (xs.max(), xs.min(), ys.max(), ys.min(), zs.max(), zs.min()) if n else None
    h = las_header(n, pdrf=pdrf, version_minor=version_minor, record_length=dt.itemsize, vlrs=vlrs,
                   has_extra=extra is not None or bool(extras), scale=sc, offset=of, bbox=bbox, by_return=byret)
    return h + recs.tobytes()


def las_header(n: int, *, pdrf: int, version_minor: int, record_length: int, vlrs: bytes, has_extra: bool, scale, offset,
               bbox, by_return) -> bytes:
    """Header and VLRs of an uncompressed LAS file of n points: bbox is
    (max x, min x, max y, min y, max z, min z) of the coordinates,
    by_return the point counts by return number 1-5."""
    header_size = 227 if version_minor <= 2 else 375
    offset_to_points = header_size + len(vlrs)
    sc, of, byret = scale, offset, by_return
    h = bytearray(header_size)
    h[0:4] = b"LASF"
    h[24], h[25] = 1, version_minor
    h[26:26 + 9] = b"synthetic"
    h[58:58 + 19] = b"potreeconverter_b200"[:19]
    struct.pack_into("<HH", h, 90, 1, 2024)
    struct.pack_into("<H", h, 94, header_size)
    struct.pack_into("<I", h, 96, offset_to_points)
    struct.pack_into("<I", h, 100, 1 if has_extra else 0)
    struct.pack_into("<B", h, 104, pdrf)
    struct.pack_into("<H", h, 105, record_length)
    struct.pack_into("<I", h, 107, n if n < 2**32 else 0)
    struct.pack_into("<5I", h, 111, *[int(v) if n < 2**32 else 0 for v in byret])
    struct.pack_into("<3d", h, 131, *sc)
    struct.pack_into("<3d", h, 155, *of)
    if n:
        struct.pack_into("<6d", h, 179, *bbox)
    if version_minor >= 4:
        struct.pack_into("<Q", h, 235, 0)
        struct.pack_into("<I", h, 243, 0)
        struct.pack_into("<Q", h, 247, n)
        struct.pack_into("<15Q", h, 255, *([int(v) for v in byret] + [0] * 10))
    return bytes(h) + vlrs


def _common_attrs(rng, n, z):
    nret = rng.integers(1, 6, n)
    ret = np.minimum(rng.integers(1, 6, n), nret)
    bits = (ret | (nret << 3)).astype(np.uint8)
    zr = (z - z.min()) / max(float(np.ptp(z)), 1e-9)
    ramp = np.stack([zr * 50000, (1 - np.abs(zr - 0.5) * 2) * 50000, (1 - zr) * 50000], 1)
    rgb = np.clip(ramp + rng.uniform(-2000, 2000, (n, 3)) + 6000, 0, 65535).astype(np.uint16)
    return {
        "intensity": rng.integers(0, 65536, n, dtype=np.uint16),
        "bits": bits,
        "classification": rng.integers(0, 32, n, dtype=np.uint8),
        "scan_angle_rank": rng.integers(-30, 31, n).astype(np.int8),
        "user_data": rng.integers(0, 256, n, dtype=np.uint8),
        "point_source_id": rng.integers(0, 64, n, dtype=np.uint16),
        "red": rgb[:, 0], "green": rgb[:, 1], "blue": rgb[:, 2],
    }


def _quantize(x):
    return np.round(np.asarray(x, dtype=np.float64) / SCALE).astype(np.int32)


def terrain(n: int, seed: int, extent: float = 500.0) -> bytes:
    """Config-0 style 2.5D terrain with facades, LAS 1.2 point format 2."""
    rng = np.random.default_rng(seed)
    n_fac = n // 10
    n_gnd = n - n_fac
    amps = rng.uniform(2.0, 10.0, 3)
    freqs = rng.uniform(0.5, 3.0, (3, 2)) * (2 * np.pi / extent)
    phases = rng.uniform(0, 2 * np.pi, 3)

    def height(x, y):
        h = np.zeros_like(x)
        for a, (fx, fy), p in zip(amps, freqs, phases):
            h += a * np.sin(fx * x + fy * y + p)
        return h

    x = rng.uniform(0, extent, n_gnd)
    y = rng.uniform(0, extent, n_gnd)
    z = height(x, y) + rng.normal(0, 0.05, n_gnd)
    # vertical facades: axis-aligned wall segments
    nwalls = max(1, n_fac // 5000 + 4)
    wx0 = rng.uniform(0.05 * extent, 0.95 * extent, nwalls)
    wy0 = rng.uniform(0.05 * extent, 0.95 * extent, nwalls)
    wlen = rng.uniform(0.02 * extent, 0.08 * extent, nwalls)
    whgt = rng.uniform(5.0, 30.0, nwalls)
    wdir = rng.integers(0, 2, nwalls)
    w = rng.integers(0, nwalls, n_fac)
    t = rng.uniform(0, 1, n_fac) * wlen[w]
    fx = np.clip(np.where(wdir[w] == 0, wx0[w] + t, wx0[w]), 0, extent)
    fy = np.clip(np.where(wdir[w] == 0, wy0[w], wy0[w] + t), 0, extent)
    fz = height(fx, fy) + rng.uniform(0, 1, n_fac) * whgt[w]
    xs = np.concatenate([x, fx])
    ys = np.concatenate([y, fy])
    zs = np.concatenate([z, fz])
    perm = rng.permutation(n)
    xs, ys, zs = xs[perm], ys[perm], zs[perm]
    X, Y, Z = _quantize(xs), _quantize(ys), _quantize(zs)
    attrs = _common_attrs(rng, n, zs)
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


def hotspots(n: int, seed: int, extent: float = 2000.0, height: float = 50.0,
             n_spots: int = 20) -> bytes:
    """Config-1 style clustered slab, LAS 1.4 point format 3 + float extra."""
    rng = np.random.default_rng(seed)
    sig = rng.uniform(5.0, 40.0, n_spots)
    cx = rng.uniform(0.1 * extent, 0.9 * extent, n_spots)
    cy = rng.uniform(0.1 * extent, 0.9 * extent, n_spots)
    # 100x background density inside each spot's 1-sigma disc
    area_bg = extent * extent
    w_spot = 100.0 * np.pi * sig ** 2
    p_bg = area_bg / (area_bg + w_spot.sum())
    n_bg = int(round(n * p_bg))
    n_sp = n - n_bg
    which = rng.choice(n_spots, n_sp, p=w_spot / w_spot.sum())
    xs = np.concatenate([rng.uniform(0, extent, n_bg), cx[which] + rng.normal(0, 1, n_sp) * sig[which]])
    ys = np.concatenate([rng.uniform(0, extent, n_bg), cy[which] + rng.normal(0, 1, n_sp) * sig[which]])
    zs = np.concatenate([rng.uniform(0, height, n_bg),
                         np.clip(height * 0.5 + rng.normal(0, 1, n_sp) * sig[which] * 0.3, 0, height)])
    xs = np.clip(xs, 0, extent)
    ys = np.clip(ys, 0, extent)
    perm = rng.permutation(n)
    xs, ys, zs = xs[perm], ys[perm], zs[perm]
    X, Y, Z = _quantize(xs), _quantize(ys), _quantize(zs)
    attrs = _common_attrs(rng, n, zs)
    attrs["gps_time"] = np.arange(n, dtype=np.float64) * 1e-4 + 3.0e5 + rng.uniform(-1e-5, 1e-5, n)
    extra = rng.normal(0, 1, n).astype(np.float32)
    return write_las(X, Y, Z, attrs, pdrf=3, version_minor=4, extra=extra)


def lattice(n: int, seed: int, cube: float = 1024.0) -> bytes:
    """Config-2 style jittered lattice with pitch = cube/1024 (level-3 spacing)."""
    rng = np.random.default_rng(seed)
    pitch = cube / 1024.0
    side_xy = 1024
    nz = max(1, int(np.ceil(n / (side_xy * side_xy))))
    idx = rng.choice(side_xy * side_xy * nz, n, replace=False) if n < side_xy * side_xy * nz else np.arange(n)
    ix = idx % side_xy
    iy = (idx // side_xy) % side_xy
    iz = idx // (side_xy * side_xy)
    X = _quantize(ix * pitch) + rng.choice([-3, -2, -1, 1, 2, 3], n)
    Y = _quantize(iy * pitch) + rng.choice([-3, -2, -1, 1, 2, 3], n)
    Z = _quantize(iz * pitch) + rng.choice([-3, -2, -1, 1, 2, 3], n)
    perm = rng.permutation(n)
    X, Y, Z = X[perm].astype(np.int32), Y[perm].astype(np.int32), Z[perm].astype(np.int32)
    attrs = _common_attrs(rng, n, Z.astype(np.float64) * SCALE)
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


def _value_noise(rng, x, y, extent, octaves=6):
    h = np.zeros_like(x)
    amp, freq, total = 1.0, 4.0 / extent, 0.0
    for _ in range(octaves):
        g = rng.uniform(0, 1, (66, 66))
        gx = np.clip(x * freq, 0, 64.999)
        gy = np.clip(y * freq, 0, 64.999)
        i0, j0 = np.floor(gx).astype(np.int64) % 65, np.floor(gy).astype(np.int64) % 65
        fx, fy = gx - np.floor(gx), gy - np.floor(gy)
        sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
        v = (g[i0, j0] * (1 - sx) * (1 - sy) + g[i0 + 1, j0] * sx * (1 - sy)
             + g[i0, j0 + 1] * (1 - sx) * sy + g[i0 + 1, j0 + 1] * sx * sy)
        h += amp * v
        total += amp
        amp *= 0.5
        freq = min(freq * 2.0, 64.0 / extent)
    return h / total


def strips(n: int, seed: int, extent: float = 20000.0, n_strips: int = 40,
           width: float = 300.0) -> bytes:
    """Config-3 style aerial strips over value-noise terrain, point format 3."""
    rng = np.random.default_rng(seed)
    centers = np.linspace(width / 2, extent - width / 2, n_strips)
    s = rng.integers(0, n_strips, n)
    xs = np.clip(centers[s] + rng.uniform(-width / 2, width / 2, n) * 1.4, 0, extent)
    ys = rng.uniform(0, extent, n)
    zs = _value_noise(np.random.default_rng(seed + 1), xs, ys, extent) * 400.0
    canopy = rng.uniform(0, 1, n) < 0.15
    zs = zs + canopy * rng.uniform(0, 30.0, n)
    X, Y, Z = _quantize(xs), _quantize(ys), _quantize(zs)
    attrs = _common_attrs(rng, n, zs)
    attrs["gps_time"] = np.arange(n, dtype=np.float64) * 1e-5 + 1.0e5
    return write_las(X, Y, Z, attrs, pdrf=3, version_minor=4)


GENERATORS = {"terrain": terrain, "hotspots": hotspots, "lattice": lattice, "strips": strips}


def generate(kind: str, n: int, seed: int, **kw) -> bytes:
    return GENERATORS[kind](n, seed, **kw)


def duplicates(n: int, seed: int, extent: float = 100.0, dup_fraction: float = 0.3,
               n_sites: int = 3) -> bytes:
    """Terrain with exact duplicate positions piled on a few sites.

    Each site holds many points with identical XYZ (and differing attributes),
    which drives the per-chunk octree into its duplicate-handling path
    (indexer.cpp:1002-1099)."""
    rng = np.random.default_rng(seed)
    n_dup = int(n * dup_fraction)
    n_base = n - n_dup
    x = rng.uniform(0, extent, n_base)
    y = rng.uniform(0, extent, n_base)
    z = np.sin(x * 0.05) * 3 + rng.normal(0, 0.05, n_base)
    site = rng.integers(0, n_sites, n_dup)
    sx, sy, sz = rng.uniform(0, extent, n_sites), rng.uniform(0, extent, n_sites), rng.uniform(0, 3, n_sites)
    xs = np.concatenate([x, sx[site]])
    ys = np.concatenate([y, sy[site]])
    zs = np.concatenate([z, sz[site]])
    perm = rng.permutation(n)
    xs, ys, zs = xs[perm], ys[perm], zs[perm]
    X, Y, Z = _quantize(xs), _quantize(ys), _quantize(zs)
    attrs = _common_attrs(rng, n, zs)
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


GENERATORS["duplicates"] = duplicates


def cube(n: int, seed: int, extent: float = 1000.0) -> bytes:
    """Uniform points filling a cube, LAS 1.2 point format 2. Every octree
    level stays volumetric, so the upper nodes gather hundreds of thousands
    of candidates even for a cloud of a few hundred thousand points."""
    rng = np.random.default_rng(seed)
    xs = rng.uniform(0, extent, n)
    ys = rng.uniform(0, extent, n)
    zs = rng.uniform(0, extent, n)
    X, Y, Z = _quantize(xs), _quantize(ys), _quantize(zs)
    attrs = _common_attrs(rng, n, zs)
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


GENERATORS["cube"] = cube


# Tile layout of ``tiles``: point format, scale and extra bytes per tile,
# tiles taken row by row over a 2 x 2 grid.
TILE_FORMATS = (2, 0, 3, 1)
TILE_SCALES = (0.001, 0.01, 0.002, 0.005)
TILE_EXTRAS = ((), (), ("amplitude",), ("amplitude", "deviation"))


def tiles(n: int, seed: int, extent: float = 400.0, origin=(652000.0, 5187000.0, 230.0),
          formats=TILE_FORMATS, scales=TILE_SCALES, extras=TILE_EXTRAS) -> list:
    """A multi-file input: one terrain with facades, cut into a 2 x 2 grid of
    tiles, each written as its own LAS file with its own point format,
    scale and offset (the tile's corner, in projected coordinates of a few
    hundred kilometres) and extra-bytes attributes. Returns the file images
    in tile order; tile k holds about n / 4 points.

    Extra-bytes attributes: ``amplitude`` (float32, N(30, 5)) and
    ``deviation`` (uint16 x 2)."""
    rng = np.random.default_rng(seed)
    amps = rng.uniform(2.0, 10.0, 3)
    freqs = rng.uniform(0.5, 3.0, (3, 2)) * (2 * np.pi / extent)
    phases = rng.uniform(0, 2 * np.pi, 3)
    x = rng.uniform(0, extent, n)
    y = rng.uniform(0, extent, n)
    z = np.zeros(n)
    for a, (fx, fy), p in zip(amps, freqs, phases):
        z += a * np.sin(fx * x + fy * y + p)
    z += rng.normal(0, 0.05, n)
    wall = rng.uniform(0, 1, n) < 0.1
    z[wall] += rng.uniform(0, 20.0, int(wall.sum()))
    attrs_all = _common_attrs(rng, n, z)
    attrs_all["gps_time"] = np.arange(n, dtype=np.float64) * 1e-4 + 2.0e5
    amplitude = rng.normal(30.0, 5.0, n).astype(np.float32)
    deviation = rng.integers(0, 4096, (n, 2)).astype(np.uint16)
    half = extent / 2.0
    tile = (x >= half).astype(np.int64) + 2 * (y >= half).astype(np.int64)
    out = []
    for k, (fmt, sc) in enumerate(zip(formats, scales)):
        sel = np.flatnonzero(tile == k)
        tx, ty = (k % 2) * half, (k // 2) * half
        off = (origin[0] + tx, origin[1] + ty, origin[2])
        X = np.round((x[sel] - tx) / sc).astype(np.int32)
        Y = np.round((y[sel] - ty) / sc).astype(np.int32)
        Z = np.round(z[sel] / sc).astype(np.int32)
        attrs = {key: v[sel] for key, v in attrs_all.items()}
        ex = []
        if "amplitude" in extras[k]:
            ex.append({"name": "amplitude", "dtype": "<f4", "values": amplitude[sel], "description": "echo amplitude"})
        if "deviation" in extras[k]:
            ex.append({"name": "deviation", "dtype": "<u2", "values": deviation[sel], "description": "pulse deviation"})
        out.append(write_las(X, Y, Z, attrs, pdrf=fmt, version_minor=4 if fmt in (1, 3) else 2,
                             scale=(sc, sc, sc), offset=off, extras=ex))
    return out


def without_points(las: bytes, pdrf: int = 2) -> bytes:
    """A LAS file image in point format pdrf without points, whose scale,
    offset and header bounding box are those of las."""
    empty = bytearray(write_las(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32), {}, pdrf=pdrf,
                                version_minor=2))
    empty[131:227] = las[131:227]
    return bytes(empty)


def sources(kind: str, n: int, seed: int, **kw) -> list:
    """File images of a multi-source input: ``tiles``; ``tiles_empty`` (tiles
    1 and 3 around a point-less format-2 file with tile 0's header box, so
    rgb is an attribute no point carries); or one image of any generator."""
    if kind == "tiles":
        return tiles(n, seed, **kw)
    if kind == "tiles_empty":
        t = tiles(n, seed, **kw)
        return [t[1], without_points(t[0]), t[3]]
    return [generate(kind, n, seed, **kw)]


def exact(n: int, seed: int) -> bytes:
    """Exact-arithmetic stress: scale 2^-8, a 256 x 256 x 16 slab whose cube
    is 256 wide, so the root spacing is exactly 2 and every coordinate,
    distance and spacing is exact in FP64. Random sites of the pitch-2
    lattice (pairs exactly one spacing apart; every child-box plane is a
    lattice plane), each with a seeded partner one quantization unit nearer
    or farther along a random axis, or at the same position."""
    rng = np.random.default_rng(seed)
    sc = 2.0 ** -8
    m = n // 2
    ix = rng.integers(0, 129, m)
    iy = rng.integers(0, 129, m)
    iz = rng.integers(0, 9, m)
    base = np.stack([ix * 512, iy * 512, iz * 512], 1).astype(np.int64)  # 2 world units = 512 quanta
    axis = rng.integers(0, 3, m)
    step = rng.choice([-1, 0, 1], m)
    partner = base.copy()
    partner[np.arange(m), axis] += step * 1
    partner = np.clip(partner, 0, [65536, 65536, 4096])
    pts = np.concatenate([base, partner, [[0, 0, 0], [65536, 65536, 0]]])[:max(n, 2)]
    perm = rng.permutation(len(pts))
    pts = pts[perm]
    X, Y, Z = (pts[:, k].astype(np.int32) for k in range(3))
    attrs = _common_attrs(rng, len(pts), Z.astype(np.float64) * sc)
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2, scale=(sc, sc, sc), offset=(0.0, 0.0, 0.0))


def shell(n: int, seed: int, extent: float = 1000.0, radius: float = 0.45) -> bytes:
    """Points on a sphere of radius `radius` x extent around the centre of
    an `extent` cube (two corner points fix the cube): the candidates of the
    upper nodes lie at almost the same distance from the node centre, so the
    poisson sampler's early exit rarely fires and its scans reach the
    10,001-check cap (30,921 candidates do at 400,000 points, seed 3)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(0, 1, (n - 2, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    c = extent / 2.0
    pts = np.concatenate([c + v * radius * extent, [[0, 0, 0], [extent, extent, extent]]])
    pts = pts[rng.permutation(n)]
    X, Y, Z = _quantize(pts[:, 0]), _quantize(pts[:, 1]), _quantize(pts[:, 2])
    attrs = _common_attrs(rng, n, pts[:, 2])
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


GENERATORS["exact"] = exact
GENERATORS["shell"] = shell


def centres(n: int, seed: int, extent: float = 1024.0, levels: int = 6) -> bytes:
    """Small balls at node centres: a uniform background plus, for levels
    0 .. levels-1, clusters of points within half a node spacing
    (extent / 128 / 2^level) of the centres of that level's nodes. Their
    candidates lie within one spacing of their node's centre, where the
    poisson sampler's early-exit bound (distance - spacing)^2 accepts them
    past conflicting points (sampler_poisson.h:127-180)."""
    rng = np.random.default_rng(seed)
    pts = [rng.uniform(0, extent, (n // 2, 3))]
    per_level = (n - n // 2) // levels
    for lvl in range(levels):
        cells = 2 ** lvl
        s = extent / 128.0 / cells
        idx = rng.integers(0, cells, (per_level, 3))
        centre = (idx + 0.5) * (extent / cells)
        d = rng.normal(0, 1, (per_level, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        r = rng.uniform(0, 0.5 * s, (per_level, 1))
        pts.append(centre + d * r)
    pts.append(np.array([[0.0, 0.0, 0.0], [extent, extent, extent]]))
    pts = np.concatenate(pts)
    pts = pts[rng.permutation(len(pts))]
    X, Y, Z = _quantize(pts[:, 0]), _quantize(pts[:, 1]), _quantize(pts[:, 2])
    attrs = _common_attrs(rng, len(pts), pts[:, 2])
    return write_las(X, Y, Z, attrs, pdrf=2, version_minor=2)


GENERATORS["centres"] = centres
