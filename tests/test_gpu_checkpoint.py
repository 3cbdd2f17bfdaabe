"""Checkpoints for an exact resume (dmph_checkpoint_write / _open): a context
opened from a checkpoint steps to the same bits as the context that wrote
it, in both builds, with free debris and with rigid bodies, on the graph path
too, across neighbour rebuilds; a restart from positions and velocities
alone (what the reference's .prof restart keeps, source/DEM-MPH.cpp:433,
:690) does not.  And the drop-in executable's --checkpoint / --resume: the
files written after a resume equal those of the uninterrupted run."""
import filecmp
import os
import subprocess

import numpy as np
import pytest

from helpers import load_scene
from dem_mph_b200 import files, scenes, solver
from dem_mph_b200.abi import FLAG_LIST_REUSE, PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "dem_mph_b200", "dem_mph")


def _by_row(g):
    t, x, v, oid = g.state()
    o = np.argsort(oid)
    return t[o], x[o], v[o]


def _same_state(a, b):
    sa, sb = a.state(), b.state()
    return all(np.array_equal(u, w) for u, w in zip(sa, sb))


@pytest.mark.parametrize("build,debris", [("fp64", "free"), ("fp64", "rigid"), ("fp32", "free"),
                                          ("fp32", "rigid"), ("fp32-graph", "rigid"), ("fp32-reuse", "rigid")])
def test_resume_is_exact(build, debris, tmp_path):
    p, typ, x, v = load_scene("small3d")
    if build.startswith("fp32"):
        p.precision = PRECISION_FP32_SPLIT
    if build == "fp32-reuse":
        # list reuse, in a shear flow whose triggers come every step or two
        p.flags |= FLAG_LIST_REUSE
        v = np.array(v, dtype=np.float64).reshape(-1, 3).copy()
        fl = np.asarray(typ) < 2
        xx = np.asarray(x, dtype=np.float64).reshape(-1, 3)
        v[fl, 0] = 1.5 + 2.0 * (xx[fl, 1] / 0.12)
    a = solver.Solver(p, typ, x, v)
    if debris == "rigid":
        s = scenes.small()
        a.set_bodies(s.body, s.body_density)
    if build.endswith("graph"):
        a.set_graph(True)
    a.step(37)
    r0 = a.info().rebuilds
    path = str(tmp_path / "a.ckpt")
    a.checkpoint(path, b"schedule")
    b, user = solver.Solver.open_checkpoint(path)
    assert user == b"schedule"
    assert _same_state(a, b)
    ia, ib = a.info(), b.info()
    assert (ia.steps, ia.rebuilds, ia.time, ia.num_bodies) == (ib.steps, ib.rebuilds, ib.time, ib.num_bodies)
    for k in (1, 12, 50):
        a.step(k)
        b.step(k)
        assert _same_state(a, b), k
    assert a.info().rebuilds > r0  # rebuilds after the resume are covered
    assert a.info().rebuilds == b.info().rebuilds
    assert a.rebuild_stats() == b.rebuild_stats()
    if build == "fp32-reuse":
        t, l = a.rebuild_stats()
        assert l < t  # triggers that kept their lists are covered
    if debris == "rigid":
        ba, bb = a.bodies(), b.bodies()
        for key in ("X", "V", "L", "q"):
            assert np.array_equal(ba[key], bb[key]), key
    a.close()
    b.close()


def test_restart_from_positions_alone_is_not_exact():
    """the .prof restart: a context created afresh from the rows' positions
    and velocities rebuilds its lists at the restart and takes another path"""
    p, typ, x, v = load_scene("small3d")
    a = solver.Solver(p, typ, x, v)
    a.step(37)
    t, xr, vr = _by_row(a)
    q = p.copy()
    q.time = a.info().time
    c = solver.Solver(q, t, xr, vr)
    a.step(63)
    c.step(63)
    ta, xa, va = _by_row(a)
    tc, xc, vc = _by_row(c)
    assert np.array_equal(ta, tc)
    assert not (np.array_equal(xa, xc) and np.array_equal(va, vc))
    a.close()
    c.close()


def test_checkpoint_refuses_a_split_step(tmp_path):
    p, typ, x, v = load_scene("small3d_fluid")
    a = solver.Solver(p, typ, x, v)
    a.step(2)
    a.step_begin()
    with pytest.raises(solver.DmphError) as e:
        a.checkpoint(str(tmp_path / "x.ckpt"))
    assert e.value.code == -1
    a.step_finish(False)
    a.checkpoint(str(tmp_path / "x.ckpt"))
    a.close()


@pytest.mark.parametrize("flags", [[], ["--fp32", "--rigid"]])
def test_drop_in_resume_writes_the_same_files(flags, tmp_path):
    s = scenes.small()
    p = s.params.copy()
    data, grid = str(tmp_path / "dem.data"), str(tmp_path / "DEM.grid")
    files.write_grid(grid, p, s.type, s.x, s.v)
    p.end_time = 60 * p.dt
    p.output_interval = 20 * p.dt
    p.vtk_output_interval = 15 * p.dt
    files.write_data_file(data, p)
    full, part = tmp_path / "full", tmp_path / "part"
    full.mkdir()
    part.mkdir()
    args = [data, grid, "p%03d.prof", "v%03d.vtk", "run.log"]
    r = subprocess.run([EXE, "--dim", "3", "--checkpoint"] + flags + args, cwd=full, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    ck = str(full / "p020.prof.ckpt")
    assert os.path.exists(ck) and os.path.exists(full / "p040.prof.ckpt")
    r = subprocess.run([EXE, "--dim", "3", "--resume", ck] + flags + args, cwd=part, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    written = sorted(f for f in os.listdir(part) if f.endswith((".prof", ".vtk")))
    # after the resume at the top of step 20: every file of the full run
    # from a later step (.prof at 40, 60; VTK at 30, 45, 60)
    later = sorted(f for f in os.listdir(full) if f.endswith((".prof", ".vtk")) and f != "output.vtk"
                   and int(f[1:4]) > 20)
    assert written == later and len(written) == 5, (written, later)
    for f in written:
        assert filecmp.cmp(full / f, part / f, shallow=False), f
