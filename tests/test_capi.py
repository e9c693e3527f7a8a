"""The C-ABI library loads and exports every function the public header declares."""
import ctypes
import os
import re

from conftest import ROOT
import manapy_b200.build as build
from manapy_b200 import _lib


def header_functions():
    txt = open(os.path.join(ROOT, "include", "manapy_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(mb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_header_symbols():
    path = build.build()
    lib = ctypes.CDLL(path)
    names = header_functions()
    assert len(names) >= 19
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers exactly the header
    assert sorted(_lib.EXPORTED) == names


def test_build_info():
    build.build()
    assert b"sm_100a" in _lib.lib().mb_build_info()
