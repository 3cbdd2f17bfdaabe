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


def test_checkpoint_open_rejects_foreign_files_without_gpu_work(tmp_path):
    """the header is read and checked before any device call: a missing file,
    a file of another kind and a truncated checkpoint head fail with DMPH_EIO
    (-4); the user-buffer limit mirrors DMPH_CHECKPOINT_USER_MAX"""
    import pytest
    with open(os.path.join(ROOT, "include", "dmph.h")) as f:
        m = re.search(r"#define DMPH_CHECKPOINT_USER_MAX (\d+)", f.read())
    assert int(m.group(1)) == solver.CHECKPOINT_USER_MAX
    foreign = tmp_path / "foreign.ckpt"
    foreign.write_bytes(b"not a checkpoint at all" * 4)
    head = tmp_path / "head.ckpt"
    head.write_bytes(b"DMPHCKPT" + bytes(8))
    for path in (tmp_path / "missing.ckpt", foreign, head):
        with pytest.raises(solver.DmphError) as e:
            solver.Solver.open_checkpoint(str(path))
        assert e.value.code == -4, str(e.value)


def test_surrogate_params_layout_matches_the_header():
    """dmph_surrogate_params_default fills the ctypes mirror field by field
    (no GPU): every default lands in its field, the last one included"""
    import ctypes as C
    from dem_mph_b200 import abi
    sp = abi.SurrogateParams()
    sp.front_tolerance = -7.0
    assert solver.lib().dmph_surrogate_params_default(C.byref(sp)) == 0
    assert (sp.substeps, sp.check_interval, sp.fallback_blocks, sp.batch, sp.pool_rows, sp.residual) == \
        (8, 50, 50, 65536, 1 << 22, 1)
    assert abs(sp.tolerance - 0.02) < 1e-15 and abs(sp.learning_rate - 1e-3) < 1e-9 and sp.seed == 1234
    assert sp.front_tolerance == 0.0
