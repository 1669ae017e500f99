"""Builds libpcgpu.so (CUDA kernels for sm_100a + host C++) and the
PotreeConverter command line front end, in-tree, with nvcc and g++.

    python -m potreeconverter_b200.build            # library + CLI
    python -m potreeconverter_b200.build --clean

FP64 arithmetic must round exactly like the reference's x86-64 build, so
device code is compiled with --fmad=false (no contracted multiply-adds) and
IEEE division/square root (nvcc's defaults with --use_fast_math off).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpcgpu.so")
CLI = os.path.join(HERE, "PotreeConverter")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "--fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O2", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O2", "-fPIC", "-std=c++17", f"-I{INCLUDE}", f"-I{CSRC}", f"-I{CUDA_HOME}/include"]

CU_SOURCES = ["radix.cu", "chunking.cu", "octree.cu", "sampling.cu", "introsort.cu", "segsort.cu", "conflicts.cu", "output.cu", "laz.cu", "pipeline.cu"]
CPP_SOURCES = ["setup.cpp", "writers.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "pcgpu.h"))
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s] + headers):
            jobs.append([NVCC] + NVCC_FLAGS + ["-c", s, "-o", o])
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out.strip():
                print(out)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lpthread"])
    cli_src = os.path.join(CSRC, "cli.cpp")
    if os.path.exists(cli_src) and _newer(CLI, [cli_src, LIB]):
        _run(["g++", "-O2", "-std=c++17", f"-I{INCLUDE}", cli_src, "-o", CLI, f"-L{HERE}", "-lpcgpu",
              "-Wl,-rpath,$ORIGIN"])
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    for p in (LIB, CLI):
        if os.path.exists(p):
            os.remove(p)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose="-v" in sys.argv))
