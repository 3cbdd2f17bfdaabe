"""The list-reuse rule of the FP32 build (dmph_rebuild.cu, decide), checked
on the FP64 oracle's own trajectory (no GPU): a small tank whose fluid starts
in a shear flow of 1.5-3.5 m/s, so that the reference's trigger fires every
step or two.  The rule keeps the lists at a trigger while every particle is
within S/2 - MARGIN/2 of its position when the lists were built (S: their
skin past MaxRadius) and remakes them otherwise, the skin of new lists 0.4 dx
when triggers come at most four steps apart.  Its claim: at every step, every
pair within MaxRadius + MARGIN was within MaxRadius + S when the lists were
built, so the lists hold every pair the passes and the neighbour counts
need.  The test replays the rule on the oracle's positions and checks the
claim pair by pair, periodic x included."""
import os
import sys

import numpy as np
from scipy.spatial import cKDTree

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from dem_mph_b200 import scenes  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402


def pairs_within(x, r, xmin, box):
    """index pairs (i < j) closer than r, periodic along x (from xmin, period
    box[0]); the other axes open"""
    y = x - (x.min(axis=0) - 1.0)
    y[:, 0] = np.mod(x[:, 0] - xmin, box[0])
    t = cKDTree(y, boxsize=[box[0], 1e9, 1e9])
    return t.query_pairs(r, output_type="ndarray")


def test_reuse_rule_keeps_every_pair_on_a_real_trajectory():
    s = scenes.small(n_debris=0)
    v = s.v.copy()
    fl = s.type < 2
    v[fl, 0] = 1.5 + 2.0 * (s.x[fl, 1] / 0.12)
    p = s.params
    o = Oracle(p, s.type, s.x, v)
    dx = p.particle_spacing
    R = 3.0 * dx            # MaxRadius of these scenes (radius ratios 3.0)
    rc = R + 0.1 * dx       # MaxRadius + MARGIN
    box = [p.domain_max[0] - p.domain_min[0]]
    ids = o.get("ParticleIndex")

    def positions():
        pid = o.get("ParticleIndex")
        out = np.empty((len(pid), 3))
        out[pid] = o.get("Position")
        return out

    x = positions()
    xL, S = x.copy(), 0.1 * dx   # lists of the creation: the MARGIN skin
    gap, last_rebuilds = 0, int(o.scalar("Rebuilds"))
    kept = full = 0
    for step in range(120):
        o.step(1)
        x = positions()
        rb = int(o.scalar("Rebuilds"))
        gap += 1
        if rb > last_rebuilds:  # the reference's trigger fired this step
            last_rebuilds = rb
            d = np.linalg.norm(x - xL, axis=1)
            d[np.abs(x[:, 0] - xL[:, 0]) > 0.5 * box[0]] = 0.0  # wrapped across x: no shift to speak of
            lim = S / 2 - 0.05 * dx - 0.001 * dx
            if lim > 0 and d.max() < lim:
                kept += 1
            else:
                full += 1
                xL, S = x.copy(), (0.4 if gap <= 4 else 0.1) * dx
            gap = 0
        # the claim at this step: pairs within rc now were within R + S at xL
        P = pairs_within(x, rc, p.domain_min[0], box)
        if len(P):
            dl = xL[P[:, 0]] - xL[P[:, 1]]
            dl[:, 0] -= box[0] * np.round(dl[:, 0] / box[0])
            assert np.linalg.norm(dl, axis=1).max() <= R + S + 1e-9, step
    o.close()
    assert kept > 10 and full > 5, (kept, full)
    assert ids is not None
