"""The drop-in executable against the reference executable built from its own
sources (oracle/_ref/DEM-MPH-2d, the unmodified 2D solver): same command
line, same input files, a short SYSU-2mm run with .prof and VTK output every
few steps; every output file must be byte-identical (FP64 build).  Also the
virial pressure of the VTK output against the oracle."""
import filecmp
import os
import subprocess
import tempfile

import numpy as np
import pytest

from helpers import GOLDEN, load_scene
from oracle.oracle import Oracle, REF_DIR
from dem_mph_b200 import files, generator, scenes, solver
from dem_mph_b200.abi import PRECISION_FP32_SPLIT

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "dem_mph_b200", "dem_mph")
REF2D = os.path.join(REF_DIR, "DEM-MPH-2d")


@pytest.mark.parametrize("name", ["sysu2mm", "small3d_st"])
def test_virial_pressure_matches_oracle(name):
    p, typ, x, v = load_scene(name)
    g = solver.Solver(p, typ, x, v)
    o = Oracle(p, typ, x, v)
    for steps in (1, 30):
        g.step(steps)
        o.step(steps)
        a, b = g.field("VirialPressure"), o.get("VirialPressure")
        assert np.array_equal(a, b) or np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), name
    q = p.copy()
    q.precision = PRECISION_FP32_SPLIT
    h = solver.Solver(q, typ, x, v)
    h.step(1)
    o2 = Oracle(p, typ, x, v)
    o2.step(1)
    # by particle id (the FP32 build may order a cell's particles its own way)
    a = h.field("VirialPressure")[np.argsort(h.state()[3])]
    b = o2.get("VirialPressure")[np.argsort(o2.get("ParticleIndex"))]
    # FP32 pressures carry the strain floor of the split precision (K * 1e-7)
    assert np.abs(a - b).max() <= 1e-3 * np.abs(b).max() + 1e-6 * p.bulk_modulus[1]
    g.close()
    h.close()


REF3D = os.path.join(REF_DIR, "DEM-MPH-3d")


def write_inputs(tmp, case):
    data = os.path.join(tmp, "dem.data")
    grid = os.path.join(tmp, "DEM.grid")
    if case == "sysu2mm_2d":
        p = files.read_data_file(os.path.join(GOLDEN, "sysu2mm", "dem.data"))
        generator.boid_to_grid(os.path.join(GOLDEN, "sysu2mm", "DEM.boid"), grid)
    else:
        s = scenes.small()
        p = s.params.copy()
        files.write_grid(grid, p, s.type, s.x, s.v)
    p.end_time = 24 * p.dt
    p.output_interval = 8 * p.dt
    p.vtk_output_interval = 12 * p.dt
    files.write_data_file(data, p)
    return data, grid


@pytest.mark.parametrize("case,ref,dim", [("sysu2mm_2d", REF2D, "2"), ("dambreak_3d", REF3D, "3")])
def test_drop_in_outputs_identical_to_reference(case, ref, dim):
    if not os.path.exists(ref):
        pytest.skip("reference executable not built")
    with tempfile.TemporaryDirectory() as tmp:
        data, grid = write_inputs(tmp, case)
        outs = {}
        for tag, cmd in (("ref", [ref]), ("ours", [EXE, "--dim", dim])):
            d = os.path.join(tmp, tag)
            os.makedirs(d)
            r = subprocess.run(cmd + [data, grid, "p%03d.prof", "v%03d.vtk", "run.log"], cwd=d,
                               capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, (tag, r.stderr[-2000:])
            outs[tag] = sorted(f for f in os.listdir(d) if f.endswith((".prof", ".vtk")))
        assert outs["ref"] == outs["ours"] and len(outs["ref"]) >= 6, outs
        assert "output.vtk" in outs["ref"]
        for f in outs["ref"]:
            a, b = os.path.join(tmp, "ref", f), os.path.join(tmp, "ours", f)
            assert filecmp.cmp(a, b, shallow=False), f


def _prof_rows(path):
    with open(path) as f:
        return f.read().splitlines()[2:]


@pytest.mark.parametrize("mode", ["sidecar", "contacts"])
def test_drop_in_rigid_bodies_equal_the_abi_run(mode):
    """Rigid debris bodies through the drop-in executable: --bodies with a
    sidecar file (per-body densities) or --rigid (bodies by contact at
    1.01 dx, type densities) gives, after 24 steps, the .prof rows of the
    same run made through the C ABI with dmph_set_bodies; and the bodies
    change the run (the rows differ from the one without bodies)."""
    with tempfile.TemporaryDirectory() as tmp:
        data, grid = write_inputs(tmp, "dambreak_3d")
        s = scenes.small()
        side = os.path.join(tmp, "DEM.bodies")
        solver.write_bodies(side, s.body, s.body_density)
        runs = {}
        for tag, extra in (("bodies", ["--bodies", side] if mode == "sidecar" else ["--rigid"]), ("plain", [])):
            d = os.path.join(tmp, tag)
            os.makedirs(d)
            r = subprocess.run([EXE, "--dim", "3"] + extra + [data, grid, "p%03d.prof", "v%03d.vtk", "run.log"],
                               cwd=d, capture_output=True, text=True, timeout=600)
            assert r.returncode == 0, (tag, r.stderr[-2000:])
            runs[tag] = _prof_rows(os.path.join(d, "p024.prof"))
        assert runs["bodies"] != runs["plain"]
        # the same through the C ABI
        p = files.read_data_file(data)
        p, typ, x, v = files.read_grid(grid, p)
        p.dim = 3
        from dem_mph_b200.abi import FLAG_ALL_NEIGHBOR_COUNTS, FLAG_WALL_DEM_COEFFS
        p.flags = FLAG_ALL_NEIGHBOR_COUNTS | FLAG_WALL_DEM_COEFFS
        if mode == "sidecar":
            body, rho = solver.read_bodies(side)
        else:
            body, rho = solver.bodies_from_contacts(p, typ, x)
            assert len(rho) == len(s.body_density)
        with solver.Solver(p, typ, x, v) as g:
            g.set_bodies(body, rho)
            g.step(24)
            t, xs, vs, _ = g.state()
            out = os.path.join(tmp, "abi.prof")
            files.write_grid(out, p, t, xs, vs, time=24 * p.dt, prof=True)
        assert _prof_rows(out) == runs["bodies"]
