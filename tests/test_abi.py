"""The C ABI library (CPU-side checks: no GPU calls).

libgrim_b200.so must exist in the package directory (built by
__graft_entry__.build()), load, and export every function that
include/grim_b200.h declares; the config struct layout of the Python
binding must match the header's field list.
"""
import ctypes
import os
import re

from grim_b200 import _lib
from grim_b200 import config as C


def test_library_exports_every_declared_symbol():
    assert os.path.exists(_lib.LIB_PATH), "build libgrim_b200.so first"
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = _lib.declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_config_struct_matches_header():
    txt = open(_lib.HEADER).read()
    body = txt[txt.index("typedef struct grim_config"):txt.index("} grim_config;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    ints, dbls = [], []
    for line in body.splitlines():
        line = line.strip().rstrip(";")
        if line.startswith("int "):
            ints += [x.strip() for x in line[4:].split(",")]
        elif line.startswith("double "):
            dbls += [x.strip() for x in line[7:].split(",")]
    assert ints == C.INT_FIELDS + ["reserved_i[%d]" % C.N_RESERVED_INT]
    assert dbls == C.DOUBLE_FIELDS + ["reserved_d[%d]" % C.N_RESERVED_DOUBLE]


def test_oracle_struct_matches_product_struct():
    from oracle import oracle as O
    assert O.INT_FIELDS == C.INT_FIELDS
    assert O.DOUBLE_FIELDS == C.DOUBLE_FIELDS
    assert ctypes.sizeof(O.OrcConfig) == ctypes.sizeof(C.GrimConfig)


def test_version_string():
    L = _lib.lib()
    assert b"sm_100a" in L.grim_version()


def _build_cpp_driver(tmp_path):
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "driver")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "include"),
           os.path.join(root, "tests", "cpp", "driver.cpp"), "-L", os.path.dirname(_lib.LIB_PATH),
           "-lgrim_b200", "-Wl,-rpath," + os.path.dirname(_lib.LIB_PATH), "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_cpp_facade_compiles_and_links(tmp_path):
    """The reference-shaped C++ facade (include/grim_b200_timestepper.hpp)
    builds and links against the library with a plain C++ compiler."""
    exe = _build_cpp_driver(tmp_path)
    assert os.path.exists(exe)
