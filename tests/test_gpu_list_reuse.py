"""List reuse (DMPH_FLAG_LIST_REUSE, FP32 split build): the Verlet lists are
kept across the reference's rebuild triggers while they provably hold every
pair within MaxRadius + MARGIN.  A small tank whose fluid starts in a shear
flow of 1.5-3.5 m/s (triggers every step or two) is run with and without the
flag and by the FP64 oracle: the triggers are the reference's, fewer of them
remake the lists, the one-step forces at a step that kept its lists match the
oracle's at the same state, and the 100-step positions stay within the FP32
build's bar.  Graph replay gives the bits of launch-by-launch stepping; the
flag is refused where it does not apply."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import FLAG_LIST_REUSE, PRECISION_FP32_SPLIT
from test_gpu_fp32 import check_one_step

pytestmark = pytest.mark.gpu


def shear_scene(n_debris=0):
    s = scenes.small(n_debris=n_debris)
    v = s.v.copy()
    fluid = s.type < 2
    v[fluid, 0] = 1.5 + 2.0 * (s.x[fluid, 1] / 0.12)
    return s, v


def fp32(params, reuse):
    q = params.copy()
    q.precision = PRECISION_FP32_SPLIT
    q.flags = FLAG_LIST_REUSE if reuse else 0
    return q


def by_row(g):
    t, x, v, oid = g.state()
    o = np.argsort(oid)
    return t[o], x[o], v[o]


def test_reuse_keeps_the_physics_and_skips_list_builds():
    s, v = shear_scene()
    a = solver.Solver(fp32(s.params, True), s.type, s.x, v)
    b = solver.Solver(fp32(s.params, False), s.type, s.x, v)
    o = Oracle(s.params, s.type, s.x, v)
    kept_checked = 0
    for _ in range(100):
        t0, l0 = a.rebuild_stats()
        a.step(1)
        b.step(1)
        o.step(1)
        t1, l1 = a.rebuild_stats()
        if kept_checked < 3 and t1 > t0 and l1 == l0 and _ > 20:
            # a step that kept its lists: the next step's forces against the
            # oracle started from this state (positions and velocities)
            _, xr, vr = by_row(a)
            q = s.params.copy()
            q.time = a.info().time
            oc = Oracle(q, s.type, xr, vr)
            check_one_step(a, oc, "kept lists", same_cells=False)
            b.step(1)
            o.step(1)
            oc.close()
            kept_checked += 1
    ta, la = a.rebuild_stats()
    tb, lb = b.rebuild_stats()
    print("triggers %d (without reuse %d, oracle %d), list builds %d" % (ta, tb, int(o.scalar("Rebuilds")), la))
    assert kept_checked == 3
    assert tb == lb and la < 0.7 * ta
    assert abs(ta - int(o.scalar("Rebuilds"))) <= 1 and abs(ta - tb) <= 1
    _, xa, va = by_row(a)
    _, xb, vb = by_row(b)
    pid = o.get("ParticleIndex")
    slot = np.empty(len(pid), np.int64)
    slot[pid] = np.arange(len(pid))
    xo = o.get("Position")[slot]
    L = float(np.ptp(xo, axis=0).max())
    assert np.abs(xa - xo).max() / L <= 1e-6 and np.abs(xb - xo).max() / L <= 1e-6
    a.close()
    b.close()
    o.close()


def test_reuse_with_rigid_bodies_graph_equals_launches():
    """debris as rigid bodies: reuse active; graph replay and launch-by-launch
    stepping give the same bits through kept and remade lists"""
    s, v = shear_scene(n_debris=3)
    runs = []
    for graph in (False, True):
        g = solver.Solver(fp32(s.params, True), s.type, s.x, v)
        g.set_bodies(s.body, s.body_density)
        g.set_graph(graph)
        g.step(60)
        runs.append((g.state(), g.bodies(), g.rebuild_stats()))
        g.close()
    (sa, ba, ra), (sb, bb, rb) = runs
    assert ra == rb and ra[1] < ra[0], (ra, rb)
    assert all(np.array_equal(u, w) for u, w in zip(sa, sb))
    assert all(np.array_equal(ba[k], bb[k]) for k in ("X", "V", "q", "L"))


def test_reuse_off_with_free_debris_and_refused_elsewhere():
    """free debris keep the reference's sort at every trigger (their DEM
    constants follow the list order), so every trigger remakes the lists; an
    ensemble and the surrogate refuse the flag"""
    s, v = shear_scene(n_debris=3)
    g = solver.Solver(fp32(s.params, True), s.type, s.x, v)
    g.step(40)
    t, l = g.rebuild_stats()
    assert t > 5 and t == l
    with pytest.raises(solver.DmphError):
        g.enable_surrogate()
    with pytest.raises(solver.DmphError):
        solver.Ensemble([g])
    g.close()


def test_reuse_at_the_benchmark_size():
    """config 2 (2.65 M particles, 200 rigid bodies) late in the flow, where
    the reference's trigger fires every step: from one state, 100 steps with
    and without list reuse take the same triggers, the reuse run remakes the
    lists at a third of them, and the fluid stays within 1e-6 of the domain
    of the run that remakes them every time"""
    s = scenes.config2()
    q = fp32(s.params, False)
    g = solver.Solver(q, s.type, s.x, s.v)
    g.set_bodies(s.body, s.body_density)
    g.set_graph(True)
    g.step(6500)
    t, x, v = by_row(g)
    time = g.info().time
    g.close()
    runs = []
    for reuse in (True, False):
        p = fp32(s.params, reuse)
        p.time = time
        h = solver.Solver(p, t, x, v)
        h.set_bodies(s.body, s.body_density)
        h.set_graph(True)
        h.step(100)
        runs.append((by_row(h), h.rebuild_stats()))
        h.close()
    (ta, xa, va), (tra, lba) = runs[0]
    (tb, xb, vb), (trb, lbb) = runs[1]
    print("config 2, 100 late steps: triggers %d / %d, list builds %d / %d" % (tra, trb, lba, lbb))
    assert abs(tra - trb) <= 1 and tra >= 80 and lba <= 0.5 * tra and lbb == trb
    fluid = ta < 2
    L = float(np.ptp(xb[fluid], axis=0).max())
    assert np.abs(xa - xb)[fluid].max() / L <= 1e-6
