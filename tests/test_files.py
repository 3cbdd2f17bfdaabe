"""Readers/writers of dem.data, .grid and .prof: the Python mirror and the
library's C++ readers agree with each other and with the reference formats."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from dem_mph_b200 import files, solver, scenes
from dem_mph_b200.abi import Params
from helpers import GOLDEN


def _params_equal(a, b):
    return bytes(a) == bytes(b)


@pytest.mark.parametrize("case", ["sysu2mm", "sysu08mm"])
def test_python_and_cpp_data_readers_agree(case):
    path = os.path.join(GOLDEN, case, "dem.data")
    inv = []
    p_py = files.read_data_file(path, invalid=inv)
    p_c = solver.read_data_file(path)
    assert _params_equal(p_py, p_c)
    assert p_py.dt == 1e-5 and p_py.radius_ratio_a == 3.0
    assert p_py.young_modulus[2] > 0 and p_py.wall_velocity[5][0] == -1.0
    # the trailing blank lines are reported as invalid, like the reference's log
    assert all(l.strip() == "" for l in inv)


def test_partial_keyword_line_assigns_prefix_like_sscanf():
    txt = "Density 1 2 3\nDt 2e-4\n"
    inv = []
    p = files.parse_data_text(txt, invalid=inv)
    assert list(p.density)[:3] == [1.0, 2.0, 3.0] and p.dt == 2e-4
    assert len(inv) == 1
    with tempfile.TemporaryDirectory() as tmp:
        fn = os.path.join(tmp, "d.data")
        with open(fn, "w") as f:
            f.write(txt)
        q = solver.read_data_file(fn)
    assert _params_equal(p, q)


def test_grid_roundtrip_and_cpp_reader():
    s = scenes.small()
    with tempfile.TemporaryDirectory() as tmp:
        g = os.path.join(tmp, "s.grid")
        files.write_grid(g, s.params, s.type, s.x, s.v)
        p1, t1, x1, v1 = files.read_grid(g)
        p2 = Params()
        t2, x2, v2 = solver.read_grid_file(g, p2)
    assert np.array_equal(t1, t2) and np.array_equal(x1, x2) and np.array_equal(v1, v2)
    assert p1.particle_spacing == p2.particle_spacing
    assert np.allclose(x1, s.x, rtol=1e-5, atol=1e-7)


def test_prof_writer_matches_python_mirror():
    s = scenes.small()
    with tempfile.TemporaryDirectory() as tmp:
        a, b = os.path.join(tmp, "a.prof"), os.path.join(tmp, "b.prof")
        p = s.params.copy()
        p.time = 1.25e-3
        files.write_grid(a, p, s.type, s.x, s.v, time=p.time, prof=True)
        x = np.ascontiguousarray(s.x)
        v = np.ascontiguousarray(s.v)
        t = np.ascontiguousarray(s.type)
        rc = solver.lib().dmph_write_prof_file(b.encode(), C.byref(p), len(t), t.ctypes.data, x.ctypes.data,
                                               v.ctypes.data)
        assert rc == 0
        assert open(a).read() == open(b).read()
        # a .prof is a valid grid input (restart)
        p3, t3, x3, v3 = files.read_grid(b)
        assert p3.time == 1.25e-3 and len(t3) == len(t)
