"""Graph replay of the step (dmph_set_graph): one CUDA graph per step, the
rebuild decision taken on the device and the rebuild run as the body of a
conditional node.  The replayed steps must give the same bits as steps
launched one kernel at a time, including the rebuilds the device decides on,
and FP64 replay must still match the oracle bit for bit."""
import numpy as np
import pytest

from helpers import load_scene
from oracle.oracle import Oracle
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu


def pair(precision, bodies):
    p, typ, x, v = load_scene("small3d")
    q = p.copy()
    q.precision = precision
    a = solver.Solver(q, typ, x, v)
    b = solver.Solver(q, typ, x, v)
    if bodies:
        s = scenes.small()
        a.set_bodies(s.body, s.body_density)
        b.set_bodies(s.body, s.body_density)
    b.set_graph(True)
    return a, b


@pytest.mark.parametrize("precision,bodies", [(0, False), (PRECISION_FP32_SPLIT, False), (PRECISION_FP32_SPLIT, True)])
def test_graph_replay_is_bit_identical(precision, bodies):
    a, b = pair(precision, bodies)
    a.step(1)
    b.step(1)
    r1 = a.info().rebuilds
    for steps in (7, 60, 80):
        a.step(steps)
        b.step(steps)
        ia, ib = a.info(), b.info()
        assert ia.rebuilds == ib.rebuilds
        assert ia.kernel_launches == ib.kernel_launches
        ta, xa, va, oa = a.state()
        tb, xb, vb, ob = b.state()
        assert np.array_equal(oa, ob) and np.array_equal(ta, tb)
        assert np.array_equal(xa, xb) and np.array_equal(va, vb)
        assert np.array_equal(a.field("Force"), b.field("Force"))
        assert np.array_equal(a.field("PressureP"), b.field("PressureP"))
        if bodies:
            ba, bb = a.bodies(), b.bodies()
            for k in ("X", "V", "q", "L"):
                assert np.array_equal(ba[k], bb[k]), k
    assert a.info().rebuilds > r1  # at least one rebuild ran inside a replayed graph
    a.close()
    b.close()


def test_graph_fp64_matches_oracle():
    p, typ, x, v = load_scene("small3d")
    g = solver.Solver(p, typ, x, v)
    g.set_graph(True)
    o = Oracle(p, typ, x, v)
    g.step(50)
    o.step(50)
    t, xg, vg, oid = g.state()
    assert np.array_equal(oid, o.get("ParticleIndex"))
    assert np.array_equal(xg, o.get("Position")) and np.array_equal(vg, o.get("Velocity"))
    assert g.info().rebuilds == int(o.scalar("Rebuilds"))
    g.close()
