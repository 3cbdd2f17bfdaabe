"""FP32 split-precision GPU path against the FP64 oracle.

Bars (the task's correctness targets for the FP32 build): per-step forces
within 1e-5, measured per particle against the sum of the magnitudes of the
force terms that make it up (pressure and viscous pair terms nearly cancel in
the interior, so an error relative to the net force is not meaningful; the
oracle reports that sum as "ForceScale"), plus the net force itself;
100-step particle positions within 1e-6 of the domain length.

The stiff equation of state P = kappa * (sum(w) - N0p) multiplies the FP32
resolution of sum(w) by the bulk modulus: positions stored relative to a cell
of width 3.1 dx carry 24 bits, so each pair distance is known to ~1e-7 and
sum(w) to ~1e-7 of N0p.  At rest in a full lattice sum(w) - N0p is 0 in FP64
and +-1e-7 N0p in FP32, which with kappa = 1e5 Pa is a pressure of 0.02 Pa
where FP64 has none.  The force check therefore has two parts: VolStrainP
within 1e-5 of N0p (the input of the pressure), and the forces within 1e-5 of
their scale once the oracle's pressure-gradient term is evaluated with the
GPU's pressures (oracle.pressure_force); the raw force difference is reported
and bounded by the strain floor.  Neighbour
sets and cell indices are still computed from FP64 positions at each rebuild
and match bit for bit; debris contacts and rigid bodies run in FP64 on FP64
master positions in this mode too.
"""
import numpy as np
import pytest

from helpers import load_scene, rel_err
from oracle.oracle import Oracle
from dem_mph_b200 import solver
from dem_mph_b200.abi import FLAG_ALL_NEIGHBOR_COUNTS, PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu

FORCE_RTOL = 1e-5


def make_pair(name):
    p, typ, x, v = load_scene(name)
    p.flags = FLAG_ALL_NEIGHBOR_COUNTS
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    return solver.Solver(q, typ, x, v), Oracle(p, typ, x, v)


def neighbour_pairs(ptr, ind, ids):
    """(particle id, neighbour id) pairs of a CSR neighbour list, sorted"""
    rows = np.repeat(ids, np.diff(ptr))
    pairs = np.stack([rows, ids[ind]], axis=1)
    return pairs[np.lexsort((pairs[:, 1], pairs[:, 0]))]


@pytest.mark.parametrize("name", ["sysu2mm", "small3d", "small3d_st", "small3d_fluid"])
def test_fp32_one_step_forces(name):
    """Neighbour sets and cells bit for bit, then the forces.  Scenes without
    free debris (small3d_fluid here) are sorted by the FP32 build's stable
    counting sort, which orders the particles inside each cell its own way,
    so arrays are compared with the oracle's by particle id."""
    g, o = make_pair(name)
    ptr, ind = g.neighbor_list()
    ids_g, ids_o = g.state()[3], o.get("ParticleIndex")
    assert np.array_equal(neighbour_pairs(ptr, ind, ids_g),
                          neighbour_pairs(o.get("NeighborPtr"), o.get("NeighborInd"), ids_o))
    check_one_step(g, o, name)
    g.close()


def check_one_step(g, o, name, same_cells=True):
    """One step of the FP32 GPU context g and the FP64 oracle o from the same
    state: cells by particle id (unless the GPU context was made with other
    cells: same_cells False), forces within FORCE_RTOL of their scale at
    equal pressures, pressures bounded by the strain and divergence
    differences, VolStrainP within FORCE_RTOL of N0p."""
    g.step(1)
    o.step(1)
    ig = np.argsort(g.state()[3])
    io = np.argsort(o.get("ParticleIndex"))

    def G(f):
        return g.field(f)[ig]

    def O(f):
        return o.get(f)[io]

    prop = O("Property")
    assert np.array_equal(g.state()[0][ig], prop)
    if same_cells:
        assert np.array_equal(G("CellIndex"), O("CellIndex"))
    fluid, solid = prop < 2, (prop >= 2) & (prop < 4)
    fg, fo = G("Force"), O("Force")
    scale = O("ForceScale") + np.linalg.norm(fo, axis=1)
    m = fluid | solid
    pg, po = G("PressureP"), O("PressureP")
    # the oracle's pressure-gradient term with the GPU's pressures (the
    # oracle takes pressures in its own slot order)
    pg_o = np.empty_like(pg)
    pg_o[io] = pg
    fo_at_pg = fo + (o.pressure_force(pg_o) - o.pressure_force(o.get("PressureP")))[io]
    err = np.linalg.norm(fg - fo_at_pg, axis=1)[m] / scale[m]
    assert np.max(err) <= FORCE_RTOL, (np.max(err), int(np.argmax(err)))
    # the pressures follow from the strain and divergence by the reference's
    # formula (kappa switched off in tension): |dP| <= K |d strain| + lambda |d div|
    bulk = np.array(list(g.params.bulk_modulus))[prop]
    bvisc = np.array(list(g.params.bulk_viscosity))[prop]
    dvs = np.abs(G("VolStrainP") - O("VolStrainP"))
    ddiv = np.abs(G("DivergenceP") - O("DivergenceP"))
    nf = fluid
    assert np.all(np.abs(pg - po)[nf] <= (bulk * dvs + bvisc * ddiv)[nf] * (1 + 1e-5) + 1e-5 * np.abs(po)[nf])
    raw = np.linalg.norm(fg - fo, axis=1)[m] / scale[m]
    print("%s: force error at equal pressures %.2e, raw %.2e (strain floor)" % (name, np.max(err), np.max(raw)))
    # VolStrainP = sum(w) - N0p cancels; compare against the sum's own scale.
    # Walls with no fluid in reach are skipped by the FP32 build's pass A (their
    # pressure is never read), so only fluid and debris particles are compared.
    vs_scale = np.abs(O("VolStrainP")).max() + 1e-300
    nw = prop < 4
    assert rel_err(G("VolStrainP")[nw], O("VolStrainP")[nw], scale=vs_scale + o.scalar("N0p")) <= FORCE_RTOL


@pytest.mark.parametrize("name", ["small3d", "sysu2mm"])
def test_fp32_hundred_steps_positions(name):
    """Fluid and wall particles after 100 steps.  Debris particles under the
    reference's per-particle DEM are left out: that contact model is not
    dissipative (its normal damping has the sign of the relative normal
    velocity times Dt, source/DEM-MPH.cpp:2601), debris bounce off the floor
    at up to 1.6 m/s in the FP64 oracle itself, and any last-bit difference is
    amplified; the FP64 build follows it bit for bit (test_gpu_parity.py) and
    the rigid-body mode used by the benchmark is compared in
    test_gpu_bodies.py."""
    g, o = make_pair(name)
    g.step(100)
    o.step(100)
    t, x, v, oid = g.state()
    xo = o.get("Position")
    L = max(np.ptp(xo, axis=0))
    # rows may be ordered differently if a rebuild fired on another step: match by original id
    order_g = np.argsort(oid)
    order_o = np.argsort(o.get("ParticleIndex"))
    keep = ~((t[order_g] >= 2) & (t[order_g] < 4))
    err = np.max(np.abs(x[order_g][keep] - xo[order_o][keep]))
    assert err <= 1e-6 * L, (err, L)
    g.close()


@pytest.mark.parametrize("name", ["small3d", "small3d_st", "sysu2mm"])
def test_verlet_list_mode_matches_stencil_mode(name):
    """The FP32 build's default Verlet-list passes against its stencil passes:
    same pairs, same per-pair arithmetic; sums differ only in how they are
    grouped (the list kernels add pairs to the FP64 sums a list batch at a
    time, the stencil kernels combine the partial sums of small chunks).
    After 40 steps a debris contact can switch on one step apart in the two
    runs (the DEM contact force is discontinuous in the gap), so from then on
    the forces compared are the fluid's."""
    p, typ, x, v = load_scene(name)
    p.precision = PRECISION_FP32_SPLIT
    a = solver.Solver(p, typ, x, v)
    b = solver.Solver(p, typ, x, v)
    b.set_pair_mode("stencil")
    # with surface tension the attractive pressure switches off at dA = N0a, a
    # discontinuity that turns last-bit differences of the sums into finite
    # force differences after a few steps: one step only there
    for steps in ((1,) if name == "small3d_st" else (1, 40)):
        a.step(steps)
        b.step(steps)
        assert a.info().rebuilds == b.info().rebuilds
        fa, fb = a.field("Force"), b.field("Force")
        tb, xb_, _, _ = b.state()
        rows = np.ones(len(fb), bool) if steps == 1 else tb < 2
        scale = np.abs(fb).max()
        d = np.abs(fa - fb).max(axis=1)
        worst = int(np.argmax(np.where(rows, d, 0)))
        assert d[rows].max() <= 1e-5 * scale, (steps, d[worst] / scale, int(tb[worst]))
        if steps == 1:
            # pass A at equal positions: the lists' walls start from the
            # wall-wall sums made at the rebuild, so only the order of the
            # FP64 additions differs (the walls included)
            for f in ("VolStrainP", "DivergenceP", "PressureP", "DensityA", "GravityCenter"):
                ga, gb = a.field(f), b.field(f)
                sc = max(np.abs(gb).max(), 1e-30)
                assert np.abs(ga - gb).max() <= 1e-6 * sc, (f, np.abs(ga - gb).max() / sc)
        _, xa, _, oa = a.state()
        _, xb, _, ob = b.state()
        L = max(np.ptp(xb, axis=0))
        assert np.array_equal(oa, ob)
        dx = np.abs(xa - xb).max(axis=1)
        assert dx[rows].max() <= 1e-6 * L, (steps, dx[rows].max() / L)
    a.close()
    b.close()


def test_fp32_drag_at_rest_on_the_cutoff_stays_finite():
    """A scene whose debris and fluid lattices put pairs exactly at RadiusP:
    FP32 rounding takes some of them in (FP64 leaves them out), and at rest the
    reference's drag expression is inf * 0 there.  The FP32 build uses the
    limit, 0, so the state stays finite."""
    import os
    import tempfile
    from dem_mph_b200 import files, scenes
    s = scenes.small(seed=3, dx=0.025)
    with tempfile.TemporaryDirectory() as tmp:
        d, g = os.path.join(tmp, "d.data"), os.path.join(tmp, "s.grid")
        files.write_data_file(d, s.params)
        files.write_grid(g, s.params, s.type, s.x, s.v)
        p = files.read_data_file(d)
        p, typ, x, v = files.read_grid(g, p)
    p.dim = 3
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, typ, x, v)
    g.step(5)
    _, xs, vs, _ = g.state()
    assert np.all(np.isfinite(xs)) and np.all(np.isfinite(vs)) and np.all(np.isfinite(g.field("Force")))
    g.close()


def test_list_stats_count_the_list_entries():
    """dmph_get_list_stats: pass B walks the fluid and debris lists, pass A
    those and the lists of walls with fluid in reach (without wall-wall
    pairs); stencil mode has no lists."""
    p, typ, x, v = load_scene("small3d")
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, typ, x, v)
    g.step(2)
    ea, eb = g.list_stats()
    t = g.state()[0]
    n_fs = int(np.sum(t < 4))
    assert 0 < eb <= ea
    assert eb >= 20 * n_fs  # a 3D lattice holds ~120 particles within the list radius
    g.set_pair_mode("stencil")
    assert g.list_stats() == (0, 0)
    g.close()


@pytest.mark.parametrize("precision", [0, PRECISION_FP32_SPLIT])
def test_list_overflow_falls_back_to_the_stencil(precision):
    """A fluid block at three times the lattice density gives lists longer
    than their capacity: the rebuild flags the overflow and the step walks the
    stencil instead, with the same bits as stencil mode (FP64 and FP32)."""
    p, typ, x, v = load_scene("small3d")
    fl = typ < 2
    h = 0.5 * p.particle_spacing
    typ3 = np.concatenate([typ, typ[fl], typ[fl]])
    x3 = np.concatenate([x, x[fl] + [h, 0.0, 0.0], x[fl] + [0.0, h, 0.0]])
    v3 = np.concatenate([v, v[fl], v[fl]])
    p.precision = precision
    a = solver.Solver(p, typ3, x3, v3)
    b = solver.Solver(p, typ3, x3, v3)
    b.set_pair_mode("stencil")
    assert a.list_stats(with_overflow=True)[2]
    a.step(1)
    b.step(1)
    for f in ("Force", "PressureP", "VolStrainP"):
        assert np.array_equal(a.field(f), b.field(f)), f
    assert np.array_equal(a.state()[1], b.state()[1])
    a.close()
    b.close()


@pytest.mark.parametrize("bodies", [False, True])
def test_debris_neighbour_counts_from_lists(bodies):
    """NeighborCount and SolidNeighborCount of the debris (the drag's solid
    fraction) come from the FP32 Verlet lists with the reference's FP64
    distance test: equal to the oracle's at the creation rebuild, and, after
    200 steps, to the FP64 stencil count of the same rebuild (the CSR list
    of dmph_get_neighbor_list, which recounts every particle that way)."""
    p, typ, x, v = load_scene("small3d")
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(q, typ, x, v)
    o = Oracle(p, typ, x, v)
    if bodies:
        from dem_mph_b200 import scenes
        s = scenes.small()
        g.set_bodies(s.body, s.body_density)
    ig, io = np.argsort(g.state()[3]), np.argsort(o.get("ParticleIndex"))
    t = g.state()[0]
    deb = (t[ig] >= 2) & (t[ig] < 4)
    for f in ("NeighborCount", "SolidNeighborCount"):
        assert np.array_equal(g.field(f)[ig][deb], o.get(f)[io][deb]), f
    g.step(200)
    assert g.info().rebuilds > 0
    nc, snc = g.field("NeighborCount"), g.field("SolidNeighborCount")
    t = g.state()[0]
    ptr, ind = g.neighbor_list()
    deb = (t >= 2) & (t < 4)
    assert np.array_equal(nc[deb], np.diff(ptr)[deb])
    solid_nb = ((t[ind] >= 2) & (t[ind] < 4)).astype(np.int64)
    snc_ref = np.add.reduceat(solid_nb, ptr[:-1]) * (np.diff(ptr) > 0)
    assert np.array_equal(snc[deb], snc_ref[deb])
    g.close()


def test_global_sums_fp64_on_the_gpu_and_fp32_error():
    """dmph_get_global_sums: the FP64 build's sums equal numpy's over its own
    state; the FP32 build's, after 100 steps, are within their error against
    the FP64 run (reported), and two calls give the same bits."""
    p, typ, x, v = load_scene("small3d_fluid")
    a = solver.Solver(p, typ, x, v)  # FP64
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    b = solver.Solver(q, typ, x, v)
    a.step(100)
    b.step(100)
    sa, sb = a.global_sums(), b.global_sums()
    sb2 = b.global_sums()
    assert all(np.array_equal(np.asarray(sb2[k]), np.asarray(sb[k])) for k in sb)
    t, xs, vs, _ = a.state()
    m = a.field("Mass")
    keep = t < 4
    mv = m[keep, None] * vs[keep]
    g = np.array(list(p.gravity))
    ref = {"mass": m[keep].sum(), "momentum": mv.sum(axis=0),
           "kinetic": 0.5 * (m[keep] * (vs[keep] ** 2).sum(axis=1)).sum(),
           "potential": -(m[keep] * (xs[keep] @ g)).sum()}
    pscale = m[keep].sum() * np.abs(vs[keep]).max()
    assert abs(sa["mass"] - ref["mass"]) <= 1e-12 * ref["mass"]
    assert np.abs(sa["momentum"] - ref["momentum"]).max() <= 1e-12 * pscale
    assert abs(sa["kinetic"] - ref["kinetic"]) <= 1e-12 * ref["kinetic"]
    assert abs(sa["potential"] - ref["potential"]) <= 1e-12 * abs(ref["potential"])
    err = {"mass": abs(sb["mass"] - sa["mass"]) / sa["mass"],
           "momentum": np.abs(sb["momentum"] - sa["momentum"]).max() / pscale,
           "kinetic": abs(sb["kinetic"] - sa["kinetic"]) / sa["kinetic"],
           "potential": abs(sb["potential"] - sa["potential"]) / abs(sa["potential"])}
    print("FP32 global sums against FP64 after 100 steps:", err)
    assert err["mass"] <= 1e-14 and err["momentum"] <= 1e-4 and err["kinetic"] <= 1e-4 and err["potential"] <= 1e-6
    a.close()
    b.close()


def test_walls_at_rest_keep_their_slots():
    """The rebuild leaves the wall slots alone when the walls are at rest and
    the counting sort is in use (rigid-body debris); this checks the
    invariant that shortcut relies on: every wall particle keeps its slot
    across rebuilds.  (The results of such runs are compared with the FP64
    oracle in test_gpu_bodies.py and by smoke.)"""
    from dem_mph_b200 import scenes
    s = scenes.small()
    p = s.params.copy()
    p.precision = PRECISION_FP32_SPLIT
    g = solver.Solver(p, s.type, s.x, s.v)
    g.set_bodies(s.body, s.body_density)
    g.step(1)
    t0, _, _, id0 = g.state()
    walls = t0 >= 4
    g.step(200)
    assert g.info().rebuilds > 1
    t1, x1, _, id1 = g.state()
    assert np.array_equal(id1[walls], id0[walls]) and np.array_equal(t1[walls], t0[walls])
    g.close()


def test_list_build_variants_change_no_result():
    """the list-build autotuner steps the scene with each launch variant of
    the list build; the states and fields must equal, bit for bit, those of
    the same steps with the default variant"""
    p, typ, x, v = load_scene("small3d")
    p.precision = PRECISION_FP32_SPLIT
    a, b = solver.Solver(p, typ, x, v), solver.Solver(p, typ, x, v)
    a.step(150)
    b.step(150)
    r0 = a.info().rebuilds
    va, ms = a.autotune_list_build(15)
    b.step(45)
    assert a.info().rebuilds - r0 >= 2 and np.sum(ms >= 0) >= 2, (a.info().rebuilds - r0, ms)
    a.set_graph(True)
    b.set_graph(True)
    a.step(30)
    b.step(30)
    sa, sb = a.state(), b.state()
    for u, w in zip(sa, sb):
        assert np.array_equal(u, w)
    for f in ("Force", "PressureP", "VolStrainP"):
        assert np.array_equal(a.field(f), b.field(f)), f
    a.close()
    b.close()
