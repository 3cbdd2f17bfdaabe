"""Failure detection during stepping: a non-finite position or velocity,
injected on the host through dmph_set_state, makes dmph_step return
DMPH_ENAN, no neighbour rebuild runs on the bad state, later calls keep
returning DMPH_ENAN, and a finite state set afterwards steps normally again.
The reference has no such check (source/errorfunc.cpp:8-31 only exits on
allocation and file errors); the fault is made on the host, never on the
GPU: no index the kernels use is derived from the injected values."""
import numpy as np
import pytest

from helpers import load_scene
from dem_mph_b200 import solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu

ENAN = -5


@pytest.mark.parametrize("prec,graph,field", [("fp64", False, "x"), ("fp32", True, "x"), ("fp32", True, "v"),
                                               ("fp32", False, "v")])
def test_nonfinite_state_is_reported(prec, graph, field):
    p, typ, x, v = load_scene("small3d")
    if prec == "fp32":
        p.precision = PRECISION_FP32_SPLIT
    with solver.Solver(p, typ, x, v) as g:
        if graph:
            g.set_graph(True)
        g.step(5)
        _, x0, v0, _ = g.state()
        fluid = np.flatnonzero(g.state()[0] < 2)
        bad_x, bad_v = x0.copy(), v0.copy()
        if field == "x":
            bad_x[fluid[len(fluid) // 2], 1] = np.nan
        else:
            bad_v[fluid[len(fluid) // 3], 0] = np.inf
        g.set_state(bad_x, bad_v)
        rb = g.info().rebuilds
        with pytest.raises(solver.DmphError) as e:
            g.step(3)
        assert e.value.code == ENAN
        assert g.info().rebuilds == rb, "a rebuild ran on a non-finite state"
        with pytest.raises(solver.DmphError) as e:
            g.step(1)
        assert e.value.code == ENAN
        # a finite state clears the flag
        g.set_state(x0, v0)
        g.step(5)
        _, x1, v1, _ = g.state()
        assert np.all(np.isfinite(x1)) and np.all(np.isfinite(v1))


def test_nonfinite_inside_a_long_call_stops_it():
    """the check inside one dmph_step call (every 256 steps) ends the call
    early: a NaN present from the first step is reported by a 600-step call"""
    p, typ, x, v = load_scene("small3d")
    p.precision = PRECISION_FP32_SPLIT
    with solver.Solver(p, typ, x, v) as g:
        g.set_graph(True)
        g.step(2)
        _, x0, v0, _ = g.state()
        bad = v0.copy()
        bad[0, 2] = np.nan
        g.set_state(x0, bad)
        steps = g.info().steps
        with pytest.raises(solver.DmphError) as e:
            g.step(600)
        assert e.value.code == ENAN
        assert g.info().steps - steps == 256
