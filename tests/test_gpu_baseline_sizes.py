"""GPU-vs-oracle parity at the benchmark's own sizes (the seeded scenes of
dem_mph_b200.scenes that bench.py times), not only on the small fixtures.

* Config 1 (186,740 particles), FP64: neighbour sets (NeighborPtr,
  NeighborInd), cell keys and permutation bit for bit, and every per-step
  field within 1e-10 of its magnitude, over steps that span a neighbour
  rebuild (calculateCellParticle / calculateNeighbor,
  source/DEM-MPH.cpp:1288-1519, 1521-1851; the pressure of
  calculatePressureP :2200-2246).
* Config 1, FP32 split: neighbour pairs by particle id, one-step forces
  within 1e-5 of their scale at equal pressures.
* Config 2 (2,645,989 particles), FP64: the creation-time cell keys and
  permutation of the reference's bitonic network at P2 = 2^22, where the
  sort runs its fused global sub-passes.
* Config 2, FP32 split: neighbour sets by particle id (an order-free hash
  per particle) and one-step forces, as for config 1.

The oracle is pinned bit for bit to the reference (test_oracle_golden.py,
test_oracle_ref.py), so agreement here is agreement with the reference.
Config 1 starts from rest and first rebuilds near step 120, so its FP64 test
starts both the GPU context and the oracle from the state the GPU reaches
after 600 steps (the flow is moving there and the reference's trigger fires
within a few steps of creation)."""
import numpy as np
import pytest

from helpers import rel_err
from oracle import oracle as orc
from oracle.oracle import Oracle
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import FLAG_ALL_NEIGHBOR_COUNTS, FLAG_WALL_DEM_COEFFS, PRECISION_FP32_SPLIT

from test_gpu_parity import compare
from test_gpu_fp32 import check_one_step, neighbour_pairs

pytestmark = pytest.mark.gpu

SEED = 1234  # the bench's scene (bench.make_scene, rank 0)


def _scene(name):
    s = scenes.config1(seed=SEED) if name == "config1" else scenes.config2(seed=SEED)
    return s.params.copy(), s.type, s.x, s.v


def _mix(z):
    """64-bit finaliser (splitmix64) of non-negative ids, wrapping"""
    z = z.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def neighbour_set_hashes(ptr, ind, ids):
    """Per particle id: the number of neighbours and an order-free hash of
    their ids (sum of mixed ids mod 2^64); equal sets give equal pairs."""
    n = len(ptr) - 1
    cnt = np.diff(ptr)
    h = np.zeros(n, np.uint64)
    chunk = 1 << 17
    with np.errstate(over="ignore"):
        for a in range(0, n, chunk):
            b = min(n, a + chunk)
            lo, hi = int(ptr[a]), int(ptr[b])
            cs = np.zeros(hi - lo + 1, np.uint64)
            np.cumsum(_mix(ids[ind[lo:hi]]), out=cs[1:])
            h[a:b] = cs[ptr[a + 1:b + 1] - lo] - cs[ptr[a:b] - lo]
    out_c = np.empty(n, np.int64)
    out_h = np.empty(n, np.uint64)
    out_c[ids] = cnt
    out_h[ids] = h
    return out_c, out_h


def test_config1_fp64_parity_across_a_rebuild():
    p, typ, x, v = _scene("config1")
    p.flags = FLAG_ALL_NEIGHBOR_COUNTS | FLAG_WALL_DEM_COEFFS
    with solver.Solver(p, typ, x, v) as s:
        s.step(600)
        _, x1, v1, oid = s.state()
        t1 = s.state()[0]
    # both start from the moving state (rows as the GPU holds them)
    g, o = solver.Solver(p, t1, x1, v1), Oracle(p, t1, x1, v1)
    try:
        compare(g, o, "creation", check_forces=False)
        ptr, ind = g.neighbor_list()
        assert np.array_equal(ptr, o.get("NeighborPtr")) and np.array_equal(ind, o.get("NeighborInd"))
        rebuilt_at = None
        for step in range(1, 61):
            g.step(1)
            o.step(1)
            if rebuilt_at is None and o.scalar("Rebuilds") >= 1:
                rebuilt_at = step
            if step in (1, 2) or (rebuilt_at is not None and step - rebuilt_at in (0, 1, 2)):
                compare(g, o, "step %d" % step)
            if rebuilt_at is not None and step - rebuilt_at >= 2:
                break
        assert rebuilt_at is not None, "no rebuild within 60 steps"
        assert g.info().rebuilds == o.scalar("Rebuilds")
        ptr, ind = g.neighbor_list()
        assert np.array_equal(ptr, o.get("NeighborPtr")) and np.array_equal(ind, o.get("NeighborInd"))
    finally:
        g.close()
        o.close()


def test_config1_fp32_pairs_and_one_step_forces():
    p, typ, x, v = _scene("config1")
    p.flags = FLAG_ALL_NEIGHBOR_COUNTS
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    g, o = solver.Solver(q, typ, x, v), Oracle(p, typ, x, v)
    try:
        ptr, ind = g.neighbor_list()
        assert np.array_equal(neighbour_pairs(ptr, ind, g.state()[3]),
                              neighbour_pairs(o.get("NeighborPtr"), o.get("NeighborInd"), o.get("ParticleIndex")))
        check_one_step(g, o, "config1")
    finally:
        g.close()
        o.close()


def test_config2_fp64_creation_sort():
    """cell keys and permutation of the creation-time bitonic sort (P2 = 2^22)"""
    p, typ, x, v = _scene("config2")
    want_key, want_perm = orc.cell_sort(p, typ, x)
    with solver.Solver(p, typ, x, v) as g:
        inf = g.info()
        assert inf.power_count == 1 << 22
        assert np.array_equal(g.field("CellIndex"), want_key)
        assert np.array_equal(g.state()[3], want_perm)


def test_config2_fp32_neighbour_sets_and_one_step_forces():
    p, typ, x, v = _scene("config2")
    p.flags = FLAG_ALL_NEIGHBOR_COUNTS
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(q, typ, x, v)
    o = Oracle(p, typ, x, v)
    try:
        ptr, ind = g.neighbor_list()
        cg, hg = neighbour_set_hashes(ptr, ind, g.state()[3])
        del ptr, ind
        co, ho = neighbour_set_hashes(o.get("NeighborPtr"), o.get("NeighborInd"), o.get("ParticleIndex"))
        assert np.array_equal(cg, co), "neighbour counts differ for %d particles" % int(np.sum(cg != co))
        assert np.array_equal(hg, ho), "neighbour sets differ for %d particles" % int(np.sum(hg != ho))
        check_one_step(g, o, "config2")
    finally:
        g.close()
        o.close()
