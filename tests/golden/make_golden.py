"""Generates tests/golden/golden.json: md5 digests of the three output files
the determinism-pinned reference converter (oracle/_ref/PotreeConverter_pinned,
built from the reference sources by oracle/Makefile) writes for seeded
synthetic inputs. Run in a container that has the reference sources:

    make -C oracle ref REF=<reference tree> && python tests/golden/make_golden.py [--multi-only | --large-only]

--multi-only keeps the single-source cases of the existing file and
regenerates the multi-source / --attributes cases. --large-only keeps every
other case and regenerates `large_cases`: the full-size workloads (the
benchmarked 50M hot-spot cloud, the 100M precision lattice, a scaled strip
cloud), whose pinned runs take tens of minutes each and run in parallel.
"""

import hashlib
import json
import os
import subprocess
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

from potreeconverter_b200 import synth  # noqa: E402

REF = os.path.join(REPO, "oracle", "_ref", "PotreeConverter_pinned")

# (case name, generator, points, seed, generator kwargs, samplers)
CASES = [
    ("terrain_200k", "terrain", 200_000, 1000, {}, ["poisson", "poisson_average", "random"]),
    ("terrain_2m", "terrain", 2_000_000, 1000, {}, ["poisson", "poisson_average", "random"]),
    ("hotspots_300k", "hotspots", 300_000, 1001, {}, ["poisson", "poisson_average", "random"]),
    ("lattice_2m", "lattice", 2_000_000, 1002, {"cube": 128.0}, ["poisson", "poisson_average", "random"]),
    ("duplicates_300k", "duplicates", 300_000, 7, {}, ["poisson", "poisson_average", "random"]),
    ("terrain_3000", "terrain", 3_000, 4, {}, ["poisson", "poisson_average", "random"]),
    ("terrain_50", "terrain", 50, 3, {}, ["poisson", "poisson_average", "random"]),
    ("exact_200k", "exact", 200_000, 3, {}, ["poisson", "poisson_average", "random"]),
    ("shell_400k", "shell", 400_000, 3, {}, ["poisson", "poisson_average", "random"]),
    ("centres_300k", "centres", 300_000, 3, {}, ["poisson", "poisson_average", "random"]),
]


# Full-size workloads: (case name, generator, points, seed, generator kwargs,
# samplers). hotspots_50m is the benchmarked cloud (50M points, LAS 1.4 point
# format 3 + float extra, 20 hot-spots, seed 1001); lattice_100m the
# precision-stress lattice (100M points, pitch = level-3 spacing, +-1-3
# quantization units of jitter, seed 1002); strips_20m a scaled instance of
# the aerial-strip cloud (seed 1003).
LARGE_CASES = [
    ("hotspots_10m", "hotspots", 10_000_000, 1001, {}, ["poisson", "poisson_average", "random"]),
    ("hotspots_50m", "hotspots", 50_000_000, 1001, {}, ["poisson", "poisson_average", "random"]),
    ("lattice_100m", "lattice", 100_000_000, 1002, {}, ["poisson"]),
    ("strips_20m", "strips", 20_000_000, 1003, {}, ["poisson", "poisson_average", "random"]),
]
LARGE_JOBS = 4  # pinned reference runs at a time (each is single-threaded)


# Inputs of several sources and --attributes lists:
# (case name, generator, points, seed, generator kwargs, source order,
#  --attributes, samplers). The "tiles" generator returns one file image per
# tile; the others one image. Source k is written as <case>_<k>.las (or
# <case>.las for one source) and the sources are passed in `order`; the
# metadata name is the first source's stem (main.cpp:146-200). Generators:
# potreeconverter_b200.synth.sources.
ALL = ["poisson", "poisson_average", "random"]
# LAZ variants: (case name, laz spec) where the spec lists the positions (in
# the passed order) of sources given as .laz, made by oracle/_ref/laz_tool
# with the vendored LASzip (chunk_size 0: LASzip's default)
LAZ = {
    "tiles_laz_200k": {"sources": [0, 1, 2, 3], "chunk_size": 0},
    "tiles_mixed_200k": {"sources": [0, 2], "chunk_size": 7000},
    "hotspots_laz_300k": {"sources": [0], "chunk_size": 9999},
}
LAZ_TOOL = os.path.join(REPO, "oracle", "_ref", "laz_tool")
MULTI_CASES = [
    ("tiles_200k", "tiles", 200_000, 11, {}, [0, 1, 2, 3], [], ALL),
    ("tiles_empty_200k", "tiles_empty", 200_000, 14, {}, [0, 1, 2], [], ALL),
    ("tiles_2m_reversed", "tiles", 2_000_000, 12, {}, [3, 2, 1, 0], [], ALL),
    ("tiles_300k_attrs", "tiles", 300_000, 13, {}, [0, 1, 2, 3],
     ["gps-time", "rgb", "return number", "no such attribute"], ALL),
    ("terrain_200k_attrs", "terrain", 200_000, 1000, {}, [0], ["rgb", "classification", "intensity"], ALL),
    ("hotspots_300k_reordered", "hotspots", 300_000, 1001, {}, [0],
     ["extra", "intensity", "return number", "number of returns", "classification", "scan angle rank",
      "user data", "point source id", "gps-time", "rgb"], ALL),
    ("tiles_laz_200k", "tiles", 200_000, 15, {}, [0, 1, 2, 3], [], ALL),
    ("tiles_mixed_200k", "tiles", 200_000, 16, {}, [2, 0, 3, 1], ["rgb", "gps-time", "intensity"], ALL),
    ("hotspots_laz_300k", "hotspots", 300_000, 17, {}, [0], [], ALL),
]


def to_laz(las: bytes, chunk_size: int, tmp: str) -> bytes:
    """The LAZ image LASzip writes for a LAS image."""
    src, dst = os.path.join(tmp, "_in.las"), os.path.join(tmp, "_out.laz")
    with open(src, "wb") as f:
        f.write(las)
    subprocess.run([LAZ_TOOL, "compress", src, dst] + ([str(chunk_size)] if chunk_size else []), check=True)
    with open(dst, "rb") as f:
        return f.read()


def multi_sources(kind, n, seed, kw, order):
    """File images of a multi-source case, in the order they are passed."""
    imgs = synth.sources(kind, n, seed, **kw)
    return [imgs[k] for k in order]


def source_names(case, kind, order):
    return [f"{case}_{k}" if kind.startswith("tiles") else case for k in order]


def md5(path):
    with open(path, "rb") as f:
        return hashlib.md5(f.read()).hexdigest()


def run_multi(tmp):
    cases = []
    for name, kind, n, seed, kw, order, attrs, methods in MULTI_CASES:
        imgs = multi_sources(kind, n, seed, kw, order)
        names = source_names(name, kind, order)
        laz = LAZ.get(name)
        paths = []
        laz_md5 = []
        for pos, (nm, img) in enumerate(zip(names, imgs)):
            if laz and pos in laz["sources"]:
                img = to_laz(img, laz["chunk_size"], tmp)
                laz_md5.append(hashlib.md5(img).hexdigest())
                paths.append(os.path.join(tmp, nm + ".laz"))
            else:
                paths.append(os.path.join(tmp, nm + ".las"))
            with open(paths[-1], "wb") as f:
                f.write(img)
        entry = {"name": name, "kind": kind, "points": n, "seed": seed, "kwargs": kw, "order": order,
                 "attributes": attrs, "meta_name": names[0],
                 "las_md5": [hashlib.md5(img).hexdigest() for img in imgs], "outputs": {}}
        if laz:
            entry["laz"] = dict(laz, laz_md5=laz_md5)
        for m in methods:
            od = os.path.join(tmp, f"{name}_{m}")
            cmd = [REF] + paths + ["-o", od, "-m", m]
            if attrs:
                cmd += ["--attributes"] + attrs
            subprocess.run(cmd, check=True, capture_output=True)
            entry["outputs"][m] = {f: {"md5": md5(os.path.join(od, f)), "size": os.path.getsize(os.path.join(od, f))}
                                   for f in ("octree.bin", "hierarchy.bin", "metadata.json")}
            print(name, m, entry["outputs"][m]["octree.bin"]["size"], flush=True)
        cases.append(entry)
    return cases


def run_large(tmp):
    """Digests of the full-size workloads; the inputs are written one at a
    time, the reference runs LARGE_JOBS at a time."""
    cases, jobs = [], []
    for name, kind, n, seed, kw, methods in LARGE_CASES:
        las = synth.generate(kind, n, seed, **kw)
        path_las = os.path.join(tmp, name + ".las")
        with open(path_las, "wb") as f:
            f.write(las)
        entry = {"name": name, "kind": kind, "points": n, "seed": seed, "kwargs": kw,
                 "las_md5": hashlib.md5(las).hexdigest(), "outputs": {}}
        del las
        cases.append(entry)
        jobs += [(entry, path_las, m) for m in methods]

    def one(job):
        entry, path_las, m = job
        od = os.path.join(tmp, f"{entry['name']}_{m}")
        subprocess.run([REF, path_las, "-o", od, "-m", m], check=True, capture_output=True)
        out = {f: {"md5": md5(os.path.join(od, f)), "size": os.path.getsize(os.path.join(od, f))}
               for f in ("octree.bin", "hierarchy.bin", "metadata.json")}
        subprocess.run(["rm", "-rf", od], check=True)
        print(entry["name"], m, out["octree.bin"]["size"], flush=True)
        return entry, m, out

    with ThreadPoolExecutor(LARGE_JOBS) as pool:
        for entry, m, out in pool.map(one, jobs):
            entry["outputs"][m] = out
    return cases


def main():
    multi_only = "--multi-only" in sys.argv
    large_only = "--large-only" in sys.argv
    path = os.path.join(HERE, "golden.json")
    out = {"generator": "potreeconverter_b200.synth", "reference": "PotreeConverter 2.0, pinned (oracle/pin/pin.h)",
           "random_seed": 1592614637, "cases": []}
    if multi_only:  # keep the single-source cases of the existing file
        with open(path) as f:
            out["cases"] = json.load(f)["cases"]
    if large_only:  # keep everything but the full-size cases
        with open(path) as f:
            out = json.load(f)
        with tempfile.TemporaryDirectory(dir=os.environ.get("GOLDEN_TMP")) as tmp:
            out["large_cases"] = run_large(tmp)
        with open(path, "w") as f:
            json.dump(out, f, indent=1)
        return
    with tempfile.TemporaryDirectory() as tmp:
        for name, kind, n, seed, kw, methods in ([] if multi_only else CASES):
            las = synth.generate(kind, n, seed, **kw)
            path_las = os.path.join(tmp, name + ".las")
            with open(path_las, "wb") as f:
                f.write(las)
            entry = {"name": name, "kind": kind, "points": n, "seed": seed, "kwargs": kw,
                     "las_md5": hashlib.md5(las).hexdigest(), "outputs": {}}
            for m in methods:
                od = os.path.join(tmp, f"{name}_{m}")
                subprocess.run([REF, path_las, "-o", od, "-m", m], check=True, capture_output=True)
                entry["outputs"][m] = {f: {"md5": md5(os.path.join(od, f)), "size": os.path.getsize(os.path.join(od, f))}
                                       for f in ("octree.bin", "hierarchy.bin", "metadata.json")}
                print(name, m, entry["outputs"][m]["octree.bin"]["size"], flush=True)
            out["cases"].append(entry)
        out["multi_cases"] = run_multi(tmp)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
