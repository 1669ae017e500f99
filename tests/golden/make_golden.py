"""Generates tests/golden/golden.json: md5 digests of the three output files
the determinism-pinned reference converter (oracle/_ref/PotreeConverter_pinned,
built from the reference sources by oracle/Makefile) writes for seeded
synthetic inputs. Run in a container that has the reference sources:

    make -C oracle ref && python tests/golden/make_golden.py
"""

import hashlib
import json
import os
import subprocess
import sys
import tempfile

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
]


def md5(path):
    with open(path, "rb") as f:
        return hashlib.md5(f.read()).hexdigest()


def main():
    out = {"generator": "potreeconverter_b200.synth", "reference": "PotreeConverter 2.0, pinned (oracle/pin/pin.h)",
           "random_seed": 1592614637, "cases": []}
    with tempfile.TemporaryDirectory() as tmp:
        for name, kind, n, seed, kw, methods in CASES:
            las = synth.generate(kind, n, seed, **kw)
            path = os.path.join(tmp, name + ".las")
            with open(path, "wb") as f:
                f.write(las)
            entry = {"name": name, "kind": kind, "points": n, "seed": seed, "kwargs": kw,
                     "las_md5": hashlib.md5(las).hexdigest(), "outputs": {}}
            for m in methods:
                od = os.path.join(tmp, f"{name}_{m}")
                subprocess.run([REF, path, "-o", od, "-m", m], check=True, capture_output=True)
                entry["outputs"][m] = {f: {"md5": md5(os.path.join(od, f)), "size": os.path.getsize(os.path.join(od, f))}
                                       for f in ("octree.bin", "hierarchy.bin", "metadata.json")}
                print(name, m, entry["outputs"][m]["octree.bin"]["size"], flush=True)
            out["cases"].append(entry)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
