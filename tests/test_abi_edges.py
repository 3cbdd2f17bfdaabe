"""Argument checks of the C ABI that run before any device work (no GPU
needed): empty and oversize particle sets, bad types, dimensions and
precisions, non-finite input, and NULL handles on every entry point."""
import ctypes as C

import numpy as np
import pytest

from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import (default_params, PRECISION_FP64, PRECISION_FP32_SPLIT)

L = solver.lib()


def create(p, typ, x, v, n=None):
    h = C.c_void_p()
    typ = np.ascontiguousarray(typ, np.int32)
    x = np.ascontiguousarray(x, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    rc = L.dmph_create(C.byref(p), len(typ) if n is None else n, typ.ctypes.data, x.ctypes.data, v.ctypes.data,
                       C.byref(h))
    return rc, h


def small():
    s = scenes.small()
    return s.params.copy(), s.type.copy(), s.x.copy(), s.v.copy()


def test_empty_and_oversize_particle_sets():
    p, t, x, v = small()
    assert create(p, t[:1], x[:1], v[:1], n=0)[0] == -1  # DMPH_EINVAL
    big = np.ones(2 ** 24 + 1, np.int32)
    assert create(p, big, x[:1], v[:1])[0] == -7  # DMPH_ERANGE, rejected before the positions are read
    assert b"2^24" in L.dmph_last_error(None)


@pytest.mark.parametrize("field,value", [("dim", 4), ("precision", 7), ("dt", 0.0), ("particle_spacing", -1.0)])
def test_bad_parameters(field, value):
    p, t, x, v = small()
    setattr(p, field, value)
    rc, h = create(p, t, x, v)
    assert rc == -1 and not h.value


def test_bad_type_and_non_finite_input():
    p, t, x, v = small()
    t2 = t.copy()
    t2[5] = 6
    assert create(p, t2, x, v)[0] == -1
    x2 = x.copy()
    x2[7, 1] = np.nan
    assert create(p, t, x2, v)[0] == -5  # DMPH_ENAN
    assert b"row 7" in L.dmph_last_error(None)
    v2 = v.copy()
    v2[3, 0] = np.inf
    assert create(p, t, x, v2)[0] == -5


def test_null_handles():
    vp = C.c_void_p(None)
    assert L.dmph_step(vp, 1) == -1
    assert L.dmph_get_info(vp, None) == -1
    assert L.dmph_set_graph(vp, 1) == -1
    assert L.dmph_set_pair_mode(vp, 1) == -1
    assert L.dmph_autotune(vp, None, None, None, None) == -1
    assert L.dmph_surrogate_collect(vp, 1) == -1
    assert L.dmph_ensemble_step(vp, 1) == -1
    assert L.dmph_destroy(vp) == 0
    assert L.dmph_ensemble_destroy(vp) == 0
    out = C.c_void_p()
    assert L.dmph_ensemble_create(None, 1, C.byref(out)) != 0
