"""dmph_cell_sort_noalloc: the allocation-free cell sort, for callers that
cannot call cudaMalloc (work recorded under stream capture, hosts whose
framework owns all device memory, real-time loops).  It must give exactly
the sorted cell keys and permutation that the solver context computes with
its own (allocated) buffers, or that the oracle's restatement of the
reference's sort gives, on repeated calls that reuse the library's
file-scope scratch array.  Collected last on purpose (file name)."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from helpers import load_scene
from dem_mph_b200 import solver

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
MAX_N = (1 << 19) - 1  # DMPH_NOALLOC_MAX_WORDS - 1


def _bind():
    L = solver.lib()
    L.dmph_cell_sort_noalloc.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
    L.dmph_last_error.restype = C.c_char_p
    L.dmph_last_error.argtypes = [C.c_void_p]
    return L


def _device_inputs(typ, x):
    import torch
    n = len(typ)
    pos = torch.tensor(np.ascontiguousarray(np.asarray(x).T), dtype=torch.float64, device="cuda")
    t = torch.tensor(np.asarray(typ), dtype=torch.int32, device="cuda")
    key = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    perm = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    return pos, t, key, perm


def _call(L, p, pos, t, key, perm, stream):
    key.fill_(-1)
    perm.fill_(-1)
    return L.dmph_cell_sort_noalloc(C.byref(p), len(t), pos.data_ptr(), t.data_ptr(), key.data_ptr(),
                                    perm.data_ptr(), stream.cuda_stream)


def _synthetic(n, seed):
    """n particles of every type scattered over the small3d tank's domain"""
    p, _, _, _ = load_scene("small3d")
    rng = np.random.default_rng(seed)
    lo, hi = np.array(p.domain_min), np.array(p.domain_max)
    x = lo + (hi - lo) * rng.random((n, 3))
    typ = rng.integers(0, 6, n).astype(np.int32)
    return p, typ, x


@pytest.mark.parametrize("name", ["small3d", "sysu2mm"])
def test_noalloc_sort_matches_context(name):
    import torch
    L = _bind()
    p, typ, x, v = load_scene(name)
    # the existing entry point: a solver context sorts the particles at creation
    with solver.Solver(p, typ, x, v) as g:
        want_key = g.field("CellIndex")
        want_perm = g.state()[3]
    pos, t, key, perm = _device_inputs(typ, x)
    stream = torch.cuda.current_stream()
    for call in range(2):
        rc = _call(L, p, pos, t, key, perm, stream)
        assert rc == 0, "call %d returned %d" % (call, rc)
        torch.cuda.synchronize()
        assert np.array_equal(key.cpu().numpy(), want_key), "keys differ on call %d" % call
        assert np.array_equal(perm.cpu().numpy(), want_perm), "permutation differs on call %d" % call


def test_noalloc_sort_largest_accepted_size():
    """n = 2^19 - 1, the padded sort exactly fills the scratch array"""
    import torch
    from oracle import oracle as orc
    L = _bind()
    p, typ, x = _synthetic(MAX_N, 11)
    want_key, want_perm = orc.cell_sort(p, typ, x)
    pos, t, key, perm = _device_inputs(typ, x)
    stream = torch.cuda.current_stream()
    for call in range(2):
        assert _call(L, p, pos, t, key, perm, stream) == 0
        torch.cuda.synchronize()
        assert np.array_equal(key.cpu().numpy(), want_key), "keys differ on call %d" % call
        assert np.array_equal(perm.cpu().numpy(), want_perm), "permutation differs on call %d" % call


def test_noalloc_sort_replayed_from_a_captured_graph():
    """one call to set up, then a call recorded under stream capture (where
    cudaMalloc is not allowed) and replayed twice on new inputs"""
    import torch
    from oracle import oracle as orc
    L = _bind()
    p, typ, x = _synthetic(20000, 5)
    pos, t, key, perm = _device_inputs(typ, x)
    assert _call(L, p, pos, t, key, perm, torch.cuda.current_stream()) == 0
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        rc = L.dmph_cell_sort_noalloc(C.byref(p), len(typ), pos.data_ptr(), t.data_ptr(), key.data_ptr(),
                                      perm.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert rc == 0, L.dmph_last_error(None)
    for seed in (6, 7):
        _, typ2, x2 = _synthetic(20000, seed)
        pos.copy_(torch.tensor(np.ascontiguousarray(x2.T), dtype=torch.float64))
        t.copy_(torch.tensor(typ2, dtype=torch.int32))
        key.fill_(-1)
        perm.fill_(-1)
        graph.replay()
        torch.cuda.synchronize()
        want_key, want_perm = orc.cell_sort(p, typ2, x2)
        assert np.array_equal(key.cpu().numpy(), want_key), "keys differ on replay (seed %d)" % seed
        assert np.array_equal(perm.cpu().numpy(), want_perm), "permutation differs on replay (seed %d)" % seed
    del graph


FRESH = r"""
import ctypes as C, sys
import numpy as np
import torch
sys.path[:0] = [%r, %r]
from dem_mph_b200 import solver
from oracle import oracle as orc
from test_zz_no_alloc import _bind, _synthetic, _device_inputs, _call
L = _bind()
p, typ, x = _synthetic(30000, 3)
pos, t, key, perm = _device_inputs(typ, x)
want_key, want_perm = orc.cell_sort(p, typ, x)
for call in range(2):
    rc = _call(L, p, pos, t, key, perm, torch.cuda.current_stream())
    assert rc == 0, (rc, L.dmph_last_error(None))
    torch.cuda.synchronize()
    assert np.array_equal(key.cpu().numpy(), want_key), call
    assert np.array_equal(perm.cpu().numpy(), want_perm), call
print("fresh ok")
"""


def test_noalloc_sort_first_call_in_a_fresh_process():
    """the set-up path: the library's first call on the device, with no
    solver context created before it"""
    r = subprocess.run([sys.executable, "-c", FRESH % (ROOT, HERE)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "fresh ok" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]


def test_noalloc_rejects_oversized_input():
    L = _bind()
    p, typ, x, v = load_scene("small3d")
    n = (1 << 19)
    rc = L.dmph_cell_sort_noalloc(C.byref(p), n, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16),
                                  C.c_void_p(16), None)
    assert rc == -7  # DMPH_ERANGE, before any device work
    assert b"DMPH_NOALLOC_MAX_WORDS" in L.dmph_last_error(None)
