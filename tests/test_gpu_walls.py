"""Moving walls (calculateWall, source/DEM-MPH.cpp:2846-2900) on the GPU: a
run that enters the 0.2-0.4 s window with a translating and spinning wall
type.  FP64 build against the oracle (itself pinned to the reference on the
same case by test_oracle_ref.py); FP32 build within the position bar; graph
replay must step the window by individual launches and give the same bits."""
import os
import tempfile

import numpy as np
import pytest

from helpers import rel_err
from oracle.oracle import Oracle
from test_oracle_ref import moving_wall_scene
from dem_mph_b200 import files, scenes, solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu


def load():
    s, params = moving_wall_scene()
    with tempfile.TemporaryDirectory() as tmp:
        d, g = os.path.join(tmp, "d.data"), os.path.join(tmp, "s.grid")
        files.write_data_file(d, params)
        files.write_grid(g, params, s.type, s.x, s.v, time=0.195)
        p = files.read_data_file(d)
        p, t, x, v = files.read_grid(g, p)
    p.dim = 3
    return p, t, x, v


def test_moving_walls_fp64_match_oracle():
    p, t, x, v = load()
    g = solver.Solver(p, t, x, v)
    o = Oracle(p, t, x, v)
    g.step(60)
    o.step(60)
    assert o.scalar("Time") > 0.2
    tg, xg, vg, og = g.state()
    assert np.array_equal(og, o.get("ParticleIndex"))
    W = max(np.ptp(o.get("Position"), axis=0))
    assert rel_err(xg, o.get("Position"), scale=W) <= 1e-13
    assert rel_err(vg, o.get("Velocity")) <= 1e-12
    walls = tg >= 4
    assert np.abs(vg[walls]).max() > 0.05  # the walls do move
    g.close()


def test_moving_walls_fp32_and_graph():
    p, t, x, v = load()
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    a = solver.Solver(q, t, x, v)
    b = solver.Solver(q, t, x, v)
    b.set_graph(True)
    o = Oracle(p, t, x, v)
    a.step(60)
    b.step(60)
    o.step(60)
    ta, xa, va, oa = a.state()
    tb, xb, vb, ob = b.state()
    assert np.array_equal(oa, ob) and np.array_equal(xa, xb) and np.array_equal(va, vb)
    xo = o.get("Position")
    L = max(np.ptp(xo, axis=0))
    ia, io = np.argsort(oa), np.argsort(o.get("ParticleIndex"))
    keep = ~((ta[ia] >= 2) & (ta[ia] < 4))  # debris: see test_gpu_fp32 (reference DEM amplifies last bits)
    assert np.abs(xa[ia][keep] - xo[io][keep]).max() <= 1e-6 * L
    a.close()
    b.close()


def test_resting_walls_keep_graph_and_lists_through_the_window():
    """Walls with zero velocity and zero angular velocity: calculateWall's
    0.2-0.4 s window moves nothing, so the FP32 build keeps its graph replay
    and its lists there (the same bits with and without the graph) and stays
    within the position bar of the FP64 oracle, which applies the window."""
    s = scenes.small(seed=14)
    params = s.params.copy()
    with tempfile.TemporaryDirectory() as tmp:
        d, g = os.path.join(tmp, "d.data"), os.path.join(tmp, "s.grid")
        files.write_data_file(d, params)
        files.write_grid(g, params, s.type, s.x, s.v, time=0.195)
        p = files.read_data_file(d)
        p, t, x, v = files.read_grid(g, p)
    p.dim = 3
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    a = solver.Solver(q, t, x, v)
    b = solver.Solver(q, t, x, v)
    b.set_graph(True)
    o = Oracle(p, t, x, v)
    a.step(60)
    b.step(60)
    o.step(60)
    assert o.scalar("Time") > 0.2
    assert not a.list_stats(with_overflow=True)[2]  # the lists stay in use
    ta, xa, va, oa = a.state()
    tb, xb, vb, ob = b.state()
    assert np.array_equal(oa, ob) and np.array_equal(xa, xb) and np.array_equal(va, vb)
    xo = o.get("Position")
    L = max(np.ptp(xo, axis=0))
    ia, io = np.argsort(oa), np.argsort(o.get("ParticleIndex"))
    keep = ~((ta[ia] >= 2) & (ta[ia] < 4))
    assert np.abs(xa[ia][keep] - xo[io][keep]).max() <= 1e-6 * L
    a.close()
    b.close()
