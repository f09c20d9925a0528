"""The C ABI: the in-tree library loads and exports every function that
include/*.h declares (no GPU needed; nothing is computed)."""
import ctypes
import os
import re

import pytest

from espreso_b200 import feti4i as F

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("feti4i.h", "feti4i_ext.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(FETI4I\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_reference_interface():
    names = declared_functions()
    for ref in ["FETI4ISetDefaultIntegerOptions", "FETI4ISetDefaultRealOptions", "FETI4ICreateStiffnessMatrix",
                "FETI4IAddElement", "FETI4ICreateInstance", "FETI4ISolve", "FETI4IUpdateStiffnessMatrix",
                "FETI4IUpdateRhs", "FETI4IUpdateDirichlet", "FETI4IDestroy"]:
        assert ref in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = ctypes.CDLL(F.LIB_PATH)
    assert hasattr(lib, name), name


def test_binding_covers_header():
    assert sorted(F.EXPORTED) == declared_functions()
