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
