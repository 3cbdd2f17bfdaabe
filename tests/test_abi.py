"""libdmph.so loads without a GPU and exports every entry point of include/dmph.h."""
import ctypes
import os
import re

from dem_mph_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            with open(os.path.join(inc, fn)) as f:
                txt = f.read()
            names |= set(re.findall(r"\b(dmph_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(solver.LIB_PATH)
    names = declared_functions()
    assert "dmph_create" in names and "dmph_step" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_string():
    assert b"sm_100a" in solver.lib().dmph_version()


def test_create_rejects_bad_input_without_gpu_work():
    """argument validation happens before any device call"""
    from dem_mph_b200.abi import default_params
    import numpy as np
    p = default_params()
    with __import__("pytest").raises(solver.DmphError):
        solver.Solver(p, np.array([9], np.int32), np.zeros((1, 3)), np.zeros((1, 3)))
