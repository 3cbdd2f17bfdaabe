"""dmph_cell_sort_noalloc: the allocation-free cell sort, for callers that
cannot call cudaMalloc (work recorded under stream capture, hosts whose
framework owns all device memory, real-time loops).  It must give exactly
the sorted cell keys and permutation that the solver context computes with
its own (allocated) buffers, on repeated calls that reuse the library's
file-scope scratch array.  Collected last on purpose (file name)."""
import ctypes as C

import numpy as np
import pytest

from helpers import load_scene
from dem_mph_b200 import solver

pytestmark = pytest.mark.gpu


def _bind():
    L = solver.lib()
    L.dmph_cell_sort_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    return L


@pytest.mark.parametrize("name", ["small3d", "sysu2mm"])
def test_noalloc_sort_matches_context(name):
    import torch
    L = _bind()
    p, typ, x, v = load_scene(name)
    # the existing entry point: a solver context sorts the particles at creation
    with solver.Solver(p, typ, x, v) as g:
        want_key = g.field("CellIndex")
        want_perm = g.state()[3]
    n = len(typ)
    pos = torch.tensor(np.ascontiguousarray(x.T), dtype=torch.float64, device="cuda")
    t = torch.tensor(typ, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    for call in range(2):
        key = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
        rc = L.dmph_cell_sort_noalloc(C.byref(p), n, pos.data_ptr(), t.data_ptr(), key.data_ptr(),
                                      perm.data_ptr(), stream.cuda_stream)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        assert np.array_equal(key.cpu().numpy(), want_key), "keys differ on call %d" % call
        assert np.array_equal(perm.cpu().numpy(), want_perm), "permutation differs on call %d" % call


def test_noalloc_rejects_oversized_input():
    L = _bind()
    p, typ, x, v = load_scene("small3d")
    n = (1 << 19)
    rc = L.dmph_cell_sort_noalloc(C.byref(p), n, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                  C.c_void_p(16), None)
    assert rc == -7  # DMPH_ERANGE, before any device work
