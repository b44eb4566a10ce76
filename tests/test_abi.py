"""The C-ABI library loads and exports every entry point include/phx.h declares
(no device calls)."""
import ctypes
import os
import re

import pytest

from phenlei_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            out |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(phx_\w+)\s*\(", txt, re.M))
    return out


def test_library_exports_all_declared_symbols():
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    lib = ctypes.CDLL(solver.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in sorted(syms) if not hasattr(lib, s)]
    assert not missing, missing


def test_default_params_match_reference_defaults():
    if not os.path.exists(solver.LIB_PATH):
        pytest.skip("libphx.so not built")
    p = solver.make_params()
    assert p.refGama == 1.4 and p.venkatCoeff == 5.0 and p.CFLVaryStep == 500
    assert p.nLUSGSSweeps == 1 and p.roeEntropyFixMethod == 3
