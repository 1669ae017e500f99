"""Seeded synthetic LAS images made on the GPU (torch), for workloads too
large for the numpy generator of ``synth``: the aerial-strip cloud of
billions of points and the jobs of the request-loop replay.

The distributions follow ``synth.strips`` and ``synth.terrain`` (the same
shapes and value ranges); the random numbers come from a torch generator
seeded per block of 2^25 points (seed * 7919 + block), so an image depends
only on (n, seed, extent) and the torch build, not on the numpy generator.
Images are written straight into page-locked host memory (the form a
caller hands to the converter for the fastest host-to-device copies).
Benchmark infrastructure: nothing in the converter imports this module.
"""

from __future__ import annotations

import numpy as np

from . import synth

BLOCK = 1 << 25
SCALE = synth.SCALE


def _u8(v, nbytes: int):
    """Little-endian bytes of the integer tensor v (values fit nbytes)."""
    import torch
    v = v.to(torch.int64)
    return torch.stack([((v >> (8 * k)) & 0xFF).to(torch.uint8) for k in range(nbytes)], dim=1)


def _f64(v):
    import torch
    return v.to(torch.float64).contiguous().view(torch.uint8).view(-1, 8)


class _Writer:
    """Collects blocks of records into a page-locked LAS image whose header
    is written last (its box and return counts need every point)."""

    def __init__(self, n: int, rec_len: int, version_minor: int, pdrf: int, host=None):
        import torch
        self.n, self.rec_len, self.version_minor, self.pdrf = n, rec_len, version_minor, pdrf
        self.header_size = 227 if version_minor <= 2 else 375
        size = self.header_size + n * rec_len
        if host is None:
            host = torch.empty(size, dtype=torch.uint8, pin_memory=True)
        assert host.numel() >= size
        self.host = host
        self.off = self.header_size
        self.mn = [None] * 3
        self.mx = [None] * 3
        self.by_return = np.zeros(5, np.int64)

    def add(self, X, Y, Z, ret, rec_bytes):
        import torch
        for a, v in enumerate((X, Y, Z)):
            lo, hi = int(v.min()), int(v.max())
            self.mn[a] = lo if self.mn[a] is None else min(self.mn[a], lo)
            self.mx[a] = hi if self.mx[a] is None else max(self.mx[a], hi)
        self.by_return += torch.bincount(ret.clamp(1, 5) - 1, minlength=5)[:5].cpu().numpy()
        nb = rec_bytes.numel()
        self.host[self.off:self.off + nb].copy_(rec_bytes.view(-1))
        self.off += nb

    def finish(self):
        import torch
        bbox = (self.mx[0] * SCALE, self.mn[0] * SCALE, self.mx[1] * SCALE, self.mn[1] * SCALE, self.mx[2] * SCALE,
                self.mn[2] * SCALE)
        h = synth.las_header(self.n, pdrf=self.pdrf, version_minor=self.version_minor, record_length=self.rec_len, vlrs=b"",
                             has_extra=False, scale=(SCALE,) * 3, offset=(0.0,) * 3, bbox=bbox, by_return=self.by_return)
        assert len(h) == self.header_size
        self.host[:len(h)].copy_(torch.frombuffer(bytearray(h), dtype=torch.uint8))
        return self.host[:self.header_size + self.n * self.rec_len]


def _common(gen, m, z, z_range, device):
    """Attributes of synth._common_attrs: returns, classification, scan
    angle, user data, source id, intensity and a height-ramp colour."""
    import torch
    nret = torch.randint(1, 6, (m,), generator=gen, device=device)
    ret = torch.minimum(torch.randint(1, 6, (m,), generator=gen, device=device), nret)
    zr = ((z - z_range[0]) / max(z_range[1] - z_range[0], 1e-9)).clamp(0, 1)
    ramp = torch.stack([zr * 50000, (1 - (zr - 0.5).abs() * 2) * 50000, (1 - zr) * 50000], 1)
    noise = torch.rand((m, 3), generator=gen, device=device, dtype=torch.float64) * 4000 - 2000
    rgb = (ramp + noise + 6000).clamp(0, 65535).to(torch.int64)
    return {
        "intensity": torch.randint(0, 65536, (m,), generator=gen, device=device),
        "bits": ret | (nret << 3), "ret": ret,
        "classification": torch.randint(0, 32, (m,), generator=gen, device=device),
        "scan_angle_rank": torch.randint(-30, 31, (m,), generator=gen, device=device) & 0xFF,
        "user_data": torch.randint(0, 256, (m,), generator=gen, device=device),
        "point_source_id": torch.randint(0, 64, (m,), generator=gen, device=device),
        "rgb": rgb,
    }


def _record(X, Y, Z, a, gps=None):
    """Point format 2 (gps None) or 3 records as an [m, 26 | 34] byte tensor."""
    import torch
    cols = [_u8(X, 4), _u8(Y, 4), _u8(Z, 4), _u8(a["intensity"], 2), _u8(a["bits"], 1), _u8(a["classification"], 1),
            _u8(a["scan_angle_rank"], 1), _u8(a["user_data"], 1), _u8(a["point_source_id"], 2)]
    if gps is not None:
        cols.append(_f64(gps))
    cols += [_u8(a["rgb"][:, 0], 2), _u8(a["rgb"][:, 1], 2), _u8(a["rgb"][:, 2], 2)]
    return torch.cat(cols, dim=1)


def _value_noise(grids, x, y, extent):
    """synth._value_noise on the device: octaves of bilinear value noise
    over 66 x 66 grids with smoothstep weights."""
    import torch
    h = torch.zeros_like(x)
    amp, freq, total = 1.0, 4.0 / extent, 0.0
    for g in grids:
        gx = (x * freq).clamp(0, 64.999)
        gy = (y * freq).clamp(0, 64.999)
        i0 = gx.floor().to(torch.int64) % 65
        j0 = gy.floor().to(torch.int64) % 65
        fx, fy = gx - gx.floor(), gy - gy.floor()
        sx, sy = fx * fx * (3 - 2 * fx), fy * fy * (3 - 2 * fy)
        v = (g[i0, j0] * (1 - sx) * (1 - sy) + g[i0 + 1, j0] * sx * (1 - sy) + g[i0, j0 + 1] * (1 - sx) * sy
             + g[i0 + 1, j0 + 1] * sx * sy)
        h += amp * v
        total += amp
        amp *= 0.5
        freq = min(freq * 2.0, 64.0 / extent)
    return h / total


def strips(n: int, seed: int, device="cuda", extent: float = 20000.0, n_strips: int = 40, width: float = 300.0, host=None):
    """Aerial strips (config-3 shape): 40 overlapping 300 m flight strips
    over 20 x 20 km, a 6-octave value-noise heightfield scaled to 0-400 m,
    15 % canopy points 0-30 m above ground; LAS 1.4 point format 3 with GPS
    time. Returns the page-locked image (a uint8 tensor)."""
    import torch
    rng = np.random.default_rng(seed + 1)
    grids = [torch.from_numpy(rng.uniform(0, 1, (66, 66))).to(device) for _ in range(6)]
    centers = torch.linspace(width / 2, extent - width / 2, n_strips, dtype=torch.float64, device=device)
    w = _Writer(n, 34, 4, 3, host)
    gen = torch.Generator(device=device)
    for b, first in enumerate(range(0, n, BLOCK)):
        m = min(BLOCK, n - first)
        gen.manual_seed(seed * 7919 + b)
        f64 = dict(generator=gen, device=device, dtype=torch.float64)
        s = torch.randint(0, n_strips, (m,), generator=gen, device=device)
        xs = (centers[s] + (torch.rand(m, **f64) * 2 - 1) * (width / 2) * 1.4).clamp(0, extent)
        ys = torch.rand(m, **f64) * extent
        zs = _value_noise(grids, xs, ys, extent) * 400.0
        canopy = torch.rand(m, **f64) < 0.15
        zs = zs + canopy * torch.rand(m, **f64) * 30.0
        X, Y, Z = [(v / SCALE).round().to(torch.int64) for v in (xs, ys, zs)]
        a = _common(gen, m, zs, (0.0, 430.0), device)
        gps = torch.arange(first, first + m, device=device, dtype=torch.float64) * 1e-5 + 1.0e5
        w.add(X, Y, Z, a["ret"], _record(X, Y, Z, a, gps))
    return w.finish()


def terrain(n: int, seed: int, extent: float = 500.0, pdrf: int = 2, device="cuda", host=None):
    """Config-0-style terrain: x, y uniform over the extent, z three seeded
    sinusoids (amplitudes 2-10 m) + N(0, 0.05 m), 10 % of the points on
    vertical facades 5-30 m tall; point format 2 (LAS 1.2) or 3 (LAS 1.4,
    GPS time). Returns the page-locked image (a uint8 tensor)."""
    import torch
    rng = np.random.default_rng(seed)
    amps = rng.uniform(2.0, 10.0, 3)
    freqs = rng.uniform(0.5, 3.0, (3, 2)) * (2 * np.pi / extent)
    phases = rng.uniform(0, 2 * np.pi, 3)
    nwalls = max(1, n // 50000 + 4)
    wx0 = torch.from_numpy(rng.uniform(0.05 * extent, 0.95 * extent, nwalls)).to(device)
    wy0 = torch.from_numpy(rng.uniform(0.05 * extent, 0.95 * extent, nwalls)).to(device)
    wlen = torch.from_numpy(rng.uniform(0.02 * extent, 0.08 * extent, nwalls)).to(device)
    whgt = torch.from_numpy(rng.uniform(5.0, 30.0, nwalls)).to(device)
    wdir = torch.from_numpy(rng.integers(0, 2, nwalls)).to(device)

    def height(x, y):
        h = torch.zeros_like(x)
        for am, (fx, fy), ph in zip(amps, freqs, phases):
            h += am * torch.sin(fx * x + fy * y + ph)
        return h

    w = _Writer(n, 26 if pdrf == 2 else 34, 2 if pdrf == 2 else 4, pdrf, host)
    gen = torch.Generator(device=device)
    for b, first in enumerate(range(0, n, BLOCK)):
        m = min(BLOCK, n - first)
        gen.manual_seed(seed * 7919 + b)
        f64 = dict(generator=gen, device=device, dtype=torch.float64)
        x = torch.rand(m, **f64) * extent
        y = torch.rand(m, **f64) * extent
        z = height(x, y) + torch.randn(m, **f64) * 0.05
        fac = torch.rand(m, **f64) < 0.1
        wi = torch.randint(0, nwalls, (m,), generator=gen, device=device)
        t = torch.rand(m, **f64) * wlen[wi]
        fx = torch.where(wdir[wi] == 0, wx0[wi] + t, wx0[wi]).clamp(0, extent)
        fy = torch.where(wdir[wi] == 0, wy0[wi], wy0[wi] + t).clamp(0, extent)
        fz = height(fx, fy) + torch.rand(m, **f64) * whgt[wi]
        x, y, z = torch.where(fac, fx, x), torch.where(fac, fy, y), torch.where(fac, fz, z)
        X, Y, Z = [(v / SCALE).round().to(torch.int64) for v in (x, y, z)]
        a = _common(gen, m, z, (-10.0, 40.0), device)
        gps = torch.arange(first, first + m, device=device, dtype=torch.float64) * 1e-4 + 3.0e5 if pdrf == 3 else None
        w.add(X, Y, Z, a["ret"], _record(X, Y, Z, a, gps))
    return w.finish()
