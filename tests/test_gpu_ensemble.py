"""Ensemble of independent scenes (dmph_ensemble_*) and the pair-pass
autotuner (dmph_autotune).  Neither has a counterpart in the reference; the
bar is that they change no result: an ensemble step must give, for every
scene, the same bits as stepping that scene alone, whatever launch variants
the tuner picked and with or without graph replay."""
import numpy as np
import pytest

from helpers import small3d_st_params
from dem_mph_b200 import scenes, solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu


MIXED = ((7, 0.02, 3, False, False), (8, 0.025, 2, True, False), (9, 0.018, 4, True, False),
         (10, 0.03, 1, False, True))
# every scene with rigid bodies or without debris: the ensemble runs its
# drifts, decisions and DEM tails as ensemble-wide launches
RIGID = ((7, 0.02, 3, True, False), (8, 0.025, 2, True, False), (9, 0.018, 4, True, False),
         (10, 0.03, 0, False, True))


def scene_list(kinds=MIXED):
    """uneven scenes: sizes, debris counts, rigid bodies on/off, surface tension on/off"""
    out = []
    for seed, dx, nd, bodies, st in kinds:
        s = scenes.small(seed=seed, dx=dx, n_debris=nd)
        p = s.params.copy()
        if st:
            p = small3d_st_params(p)
        p.precision = PRECISION_FP32_SPLIT
        out.append((s, p, bodies))
    return out


def make(items):
    sv = []
    for s, p, bodies in items:
        g = solver.Solver(p, s.type, s.x, s.v)
        if bodies:
            g.set_bodies(s.body, s.body_density)
        sv.append(g)
    return sv


def same_state(a, b):
    ta, xa, va, oa = a.state()
    tb, xb, vb, ob = b.state()
    return (np.array_equal(oa, ob) and np.array_equal(ta, tb) and np.array_equal(xa, xb)
            and np.array_equal(va, vb) and np.array_equal(a.field("PressureP"), b.field("PressureP")))


@pytest.mark.parametrize("graph,mode,kinds", [(True, "list", "mixed"), (False, "list", "mixed"),
                                              (True, "stencil", "mixed"), (True, "list", "rigid"),
                                              (False, "list", "rigid")])
def test_ensemble_matches_scenes_stepped_alone(graph, mode, kinds):
    items = scene_list(RIGID if kinds == "rigid" else MIXED)
    alone = make(items)
    members = make(items)
    for g in alone + members:
        g.set_pair_mode(mode)
    ens = solver.Ensemble(members)
    ens.set_graph(graph)
    assert len({g.n for g in members}) == len(members)  # uneven sizes
    chunks = (1, 9, 50, 140) if kinds == "rigid" else (1, 9, 50)  # rigid bodies rebuild less often
    for steps in chunks:
        for g in alone:
            g.step(steps)
        ens.step(steps)
        for k, (a, b) in enumerate(zip(alone, members)):
            assert a.info().rebuilds == b.info().rebuilds, k
            assert same_state(a, b), k
            if getattr(a, "nbodies", 0):
                ba, bb = a.bodies(), b.bodies()
                assert all(np.array_equal(ba[q], bb[q]) for q in ("X", "V", "q", "L")), k
    assert sum(g.info().rebuilds for g in members) > len(members)
    assert ens.info()["steps"] == sum(chunks)
    if kinds == "rigid" and graph:
        # fused: per recorded step, 2 head + 6 list-pass + 2 + 3 per DEM substep launches
        l0 = ens.info()["kernel_launches"]
        ens.step(4)
        assert ens.info()["kernel_launches"] - l0 == 4 * (2 + 6 + 2 + 3 * 2)
    ens.close()
    for g in alone + members:
        g.close()


def test_autotuned_variants_change_no_result():
    items = scene_list()[:2]
    ref = make(items)
    tuned = make(items)
    ens = solver.Ensemble(tuned)
    for g in ref:
        g.step(5)
    ens.step(5)
    va, vb, ma, mb = ens.autotune()
    assert 0 <= va < solver.PASS_VARIANTS and 0 <= vb < solver.PASS_VARIANTS
    assert np.all(ma > 0) and np.all(mb > 0)
    for g in ref:
        g.step(30)
    ens.step(30)
    for a, b in zip(ref, tuned):
        assert same_state(a, b)
    ens.close()
    # single-scene tuner, and every variant forced in turn, in both pair modes
    a, b = ref[0], tuned[0]
    ta, tb, ma, mb = b.autotune()  # list mode: the list-pass variants
    assert 0 <= ta < solver.LIST_VARIANTS and np.all(ma[:solver.LIST_VARIANTS] > 0)
    for v in range(solver.LIST_VARIANTS):
        b.set_variants(v, (v + 2) % solver.LIST_VARIANTS)
        a.step(3)
        b.step(3)
        assert same_state(a, b), v
    a.set_pair_mode("stencil")
    b.set_pair_mode("stencil")
    b.autotune()
    for v in range(solver.PASS_VARIANTS):
        b.set_variants(v, (v + 2) % solver.PASS_VARIANTS)
        a.step(3)
        b.step(3)
        assert same_state(a, b), v
    for g in ref + tuned:
        g.close()


def test_ensemble_rejects_fp64_and_duplicates():
    s = scenes.small()
    g = solver.Solver(s.params, s.type, s.x, s.v)  # FP64 parity build
    with pytest.raises(solver.DmphError):
        solver.Ensemble([g])
    p = s.params.copy()
    p.precision = PRECISION_FP32_SPLIT
    h = solver.Solver(p, s.type, s.x, s.v)
    with pytest.raises(solver.DmphError):
        solver.Ensemble([h, h])
    with pytest.raises(solver.DmphError):
        g.autotune()
    g.close()
    h.close()


def test_ensemble_profiling_times_the_passes_and_changes_nothing():
    """phase times of the shared pass launches, one pass A and one pass B
    per step, and the same bits as graph replay"""
    items = scene_list(RIGID)
    a, b = make(items), make(items)
    ea, eb = solver.Ensemble(a), solver.Ensemble(b)
    ea.step(5)
    eb.step(5)
    ea.set_profiling(True)
    ea.step(12)
    eb.step(12)
    ph = ea.phase_times()
    assert set(ph) == {"pass_a", "pass_b"} and ph["pass_a"][1] == 12 and ph["pass_b"][1] == 12
    assert ph["pass_a"][0] > 0 and ph["pass_b"][0] > 0
    ea.set_profiling(False)
    for x, y in zip(a, b):
        assert same_state(x, y)
    ea.close()
    eb.close()
    for g in a + b:
        g.close()
