"""Live pin of the oracle restatement against the reference solver built from
its own source (oracle/_ref).  Skipped where oracle/_ref was not built."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from dem_mph_b200 import files, scenes
from helpers import small3d_st_params
from oracle.oracle import Oracle, read_ref_dump, REF_DIR

EXE3 = os.path.join(REF_DIR, "ref_dump3d")


@pytest.mark.skipif(not os.path.exists(EXE3), reason="oracle/_ref not built (reference tree absent)")
@pytest.mark.parametrize("seed,yaw,st", [(11, False, False), (12, True, False), (13, False, True)])
def test_oracle_bit_exact_vs_reference(seed, yaw, st):
    """every array the harness dumps, the virial pressure of the output
    cadence included; st: surface tension with non-zero interaction ratios"""
    s = scenes.small(seed=seed, yaw=yaw)
    params = small3d_st_params(s.params) if st else s.params
    with tempfile.TemporaryDirectory() as tmp:
        data, grid = os.path.join(tmp, "d.data"), os.path.join(tmp, "s.grid")
        files.write_data_file(data, params)
        files.write_grid(grid, params, s.type, s.x, s.v)
        subprocess.run([EXE3, data, grid, os.path.join(tmp, "out"), "60", "60"], check=True, capture_output=True)
        ref = read_ref_dump(os.path.join(tmp, "out", "step60"))
        p = files.read_data_file(data)
        p, typ, x, v = files.read_grid(grid, p)
    p.dim = 3
    o = Oracle(p, typ, x, v)
    o.step(60)
    for k, a in ref.items():
        if k == "meta":
            continue
        b = o.get(k)
        if k == "NeighborPtr":
            a = a[:len(b)]
        assert a.shape == b.shape, k
        assert np.array_equal(a, b, equal_nan=True) if a.dtype.kind == "f" else np.array_equal(a, b), k


def moving_wall_scene(seed=14):
    """small dam break starting at t = 0.195 s, so the moving-wall window of
    calculateWall (0.2 <= Time <= 0.4, :2860) opens after ~20 steps, with the
    wall type translating and spinning (WallRotation from Omega Dt, :1166)"""
    s = scenes.small(seed=seed)
    p = s.params.copy()
    p.wall_center[4][0], p.wall_center[4][1], p.wall_center[4][2] = 0.3, 0.1, 0.15
    p.wall_velocity[4][0], p.wall_velocity[4][1] = 0.05, 0.02
    p.wall_omega[4][2] = 0.3
    return s, p


@pytest.mark.skipif(not os.path.exists(EXE3), reason="oracle/_ref not built (reference tree absent)")
def test_oracle_bit_exact_vs_reference_moving_walls():
    s, params = moving_wall_scene()
    with tempfile.TemporaryDirectory() as tmp:
        data, grid = os.path.join(tmp, "d.data"), os.path.join(tmp, "s.grid")
        files.write_data_file(data, params)
        files.write_grid(grid, params, s.type, s.x, s.v, time=0.195)
        subprocess.run([EXE3, data, grid, os.path.join(tmp, "out"), "60", "60"], check=True, capture_output=True)
        ref = read_ref_dump(os.path.join(tmp, "out", "step60"))
        p = files.read_data_file(data)
        p, typ, x, v = files.read_grid(grid, p)
    assert abs(p.time - 0.195) < 1e-12
    p.dim = 3
    o = Oracle(p, typ, x, v)
    o.step(60)
    assert o.scalar("Time") > 0.2
    for k, a in ref.items():
        if k == "meta":
            continue
        b = o.get(k)
        if k == "NeighborPtr":
            a = a[:len(b)]
        assert a.shape == b.shape, k
        assert np.array_equal(a, b, equal_nan=True) if a.dtype.kind == "f" else np.array_equal(a, b), k
