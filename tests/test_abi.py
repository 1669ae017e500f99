"""The C ABI library loads and exports every symbol include/pcgpu.h declares
(no GPU needed), and the package refuses to run without it."""

import os
import re

import pytest

import potreeconverter_b200 as pc

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(REPO, "include", "pcgpu.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)  # drop comments
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(pcg_[a-z_]+)\(", text, flags=re.M)))


def test_header_and_package_agree():
    assert declared_symbols() == sorted(pc.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = pc.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_status_strings():
    lib = pc.load_library()
    assert lib.pcg_status_string(0) == b"ok"
    assert lib.pcg_status_string(2) == b"point outside bounding box"


def test_missing_library_fails_loudly(tmp_path):
    import importlib
    saved = pc._lib
    try:
        pc._lib = None
        with pytest.raises(RuntimeError):
            pc.load_library(str(tmp_path / "missing.so"))
    finally:
        pc._lib = saved


def test_binding_structs_match_the_header(tmp_path):
    # every field of the ctypes mirrors sits at the offset the C compiler
    # gives it in include/pcgpu.h, and the structs have the same size
    import ctypes
    import subprocess
    structs = {"pcg_opts": pc._Opts, "pcg_source": pc._Source, "pcg_job": pc._Job, "pcg_stats": pc._Stats,
               "pcg_node": pc._Node, "pcg_result": pc._Result, "pcg_chunk": pc._Chunk, "pcg_octree_node": pc._OctreeNode,
               "pcg_octree_part": pc._Part}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pcgpu.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} sizeof() %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I" + os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = 0
    for line in filter(None, out):
        cname, what, value = line.split()
        py = structs[cname]
        got = ctypes.sizeof(py) if what == "sizeof()" else getattr(py, what).offset
        assert got == int(value), (cname, what)
        seen += 1
    assert seen == sum(len(p._fields_) + 1 for p in structs.values())
