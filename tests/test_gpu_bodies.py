"""Rigid debris bodies on the GPU (DMPH_FLAG_RIGID_CLUMPS mode, set through
dmph_set_bodies) against the oracle's FP64 restatement of the same model.
The mode has no reference counterpart (parity unpinned); the oracle's
conservation tests (test_bodies_oracle.py) are its physical pins.  The GPU
reduces each body's force and torque with warp shuffles, so sums differ from
the oracle's sequential sums at the last bits; the bars below allow for that
and for the FP32 build's fluid forces."""
import numpy as np
import pytest

from helpers import load_scene, rel_err
from oracle.oracle import Oracle
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu


def make(precision=0):
    p, typ, x, v = load_scene("small3d")
    s = scenes.small()
    q = p.copy()
    q.precision = precision
    g = solver.Solver(q, typ, x, v)
    o = Oracle(p, typ, x, v)
    g.set_bodies(s.body, s.body_density)
    o.set_bodies(s.body, s.body_density)
    return g, o


@pytest.mark.parametrize("precision,tol", [(0, 1e-9), (PRECISION_FP32_SPLIT, 2e-4)])
def test_bodies_match_oracle(precision, tol):
    g, o = make(precision)
    b0 = g.bodies()
    ob = o.bodies()
    assert np.allclose(b0["X"], ob["X"], rtol=0, atol=1e-12) and np.allclose(b0["M"], ob["M"])
    for steps in (1, 40):
        g.step(steps)
        o.step(steps)
        gb, ob = g.bodies(), o.bodies()
        L = 0.6
        assert np.max(np.abs(gb["X"] - ob["X"])) <= tol * L
        assert rel_err(gb["V"], ob["V"]) <= tol * 10
        assert np.max(np.abs(gb["q"] - ob["q"])) <= tol * 10
    # particles of the bodies sit where the bodies put them
    t, x, v, oid = g.state()
    xo = o.get("Position")
    order_g, order_o = np.argsort(oid), np.argsort(o.get("ParticleIndex"))
    solid = (t[order_g] >= 2) & (t[order_g] < 4)
    assert np.max(np.abs(x[order_g][solid] - xo[order_o][solid])) <= tol * 0.6
    g.close()


def test_bodies_fall_rigidly():
    """after many steps every body's particles keep their mutual distances"""
    g, _ = make(0)
    t0, x0, _, oid0 = g.state()
    g.step(60)
    t1, x1, _, oid1 = g.state()
    s = scenes.small()
    a = x0[np.argsort(oid0)]
    b = x1[np.argsort(oid1)]
    for k in range(len(s.body_density)):
        idx = np.where(s.body == k)[0]
        da = np.linalg.norm(a[idx[:, None]] - a[idx[None, :]], axis=2)
        db = np.linalg.norm(b[idx[:, None]] - b[idx[None, :]], axis=2)
        assert np.max(np.abs(da - db)) <= 1e-12
    bd = g.bodies()
    assert np.all(np.isfinite(bd["X"])) and np.all(np.abs(np.linalg.norm(bd["q"], axis=1) - 1) < 1e-12)
    g.close()
