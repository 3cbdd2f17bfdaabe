"""Shared helpers of the test-suite: golden scenes and comparisons."""
import json
import os
import tempfile

import numpy as np

from dem_mph_b200 import files, generator, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

with open(os.path.join(GOLDEN, "golden.json")) as _f:
    GOLD = json.load(_f)


def small3d_st_params(p):
    """small3d with the surface-tension model switched on (same as make_golden)."""
    q = p.copy()
    q.surface_tension[1] = 0.072
    q.surface_tension[2] = 0.03
    for a, b, r in ((1, 1, 1.0), (1, 2, 0.4), (2, 1, 0.6), (1, 4, 0.2), (4, 1, 0.3), (2, 2, 0.5)):
        q.interaction_ratio[a][b] = r
    return q


def load_scene(name):
    """(params, type, x, v) of a golden scene, read back from the same text
    files the reference read (positions carry the grid file's %e rounding)."""
    with tempfile.TemporaryDirectory() as tmp:
        data = os.path.join(tmp, "dem.data")
        grid = os.path.join(tmp, "scene.grid")
        if name.startswith("sysu"):
            tag = "sysu2mm" if name == "sysu2mm" else "sysu08mm"
            d = os.path.join(GOLDEN, tag)
            with open(os.path.join(d, "dem.data")) as f, open(data, "w") as g:
                g.write(f.read())
            generator.boid_to_grid(os.path.join(d, "DEM.boid"), grid)
            dim = 2
        else:
            # small3d_fluid: the same tank and column without debris
            s = scenes.small(n_debris=0) if name == "small3d_fluid" else scenes.small()
            p = small3d_st_params(s.params) if name == "small3d_st" else s.params
            files.write_data_file(data, p)
            files.write_grid(grid, p, s.type, s.x, s.v)
            dim = 3
        p = files.read_data_file(data)
        p, typ, x, v = files.read_grid(grid, p)
    p.dim = dim
    return p, typ, x, v


def fingerprint_ok(arr, fp, rtol=1e-12):
    """Compare an array with a golden fingerprint; returns (ok, message)."""
    a = np.asarray(arr)
    if a.size != fp["n"]:
        return False, "size %d != %d" % (a.size, fp["n"])
    if "sha256" in fp:
        import hashlib
        h = hashlib.sha256(np.ascontiguousarray(a.astype(fp["dtype"])).tobytes()).hexdigest()
        return h == fp["sha256"], "sha256 differs"
    f = a.astype(np.float64).ravel()
    w = (np.arange(f.size) % 97 + 1).astype(np.float64)
    nan = int(np.sum(np.isnan(f)))
    if nan != fp["nan"]:
        return False, "nan count %d != %d" % (nan, fp["nan"])
    absum = float(np.nansum(np.abs(f)))
    scale = max(abs(fp["abs"]), 1e-300)
    for key, val in (("sum", float(np.nansum(f))), ("abs", absum), ("wsum", float(np.nansum(f * w)))):
        ref = fp[key]
        tol = rtol * (scale if key != "wsum" else scale * 97)
        if not (abs(val - ref) <= tol or (np.isnan(val) and np.isnan(ref))):
            return False, "%s %.17g != %.17g" % (key, val, ref)
    return True, ""


def rel_err(a, b, scale=None):
    """max |a-b| / scale, with scale = max|b| by default (forces near-cancel,
    so errors are measured against the field's magnitude, not per element)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    s = scale if scale is not None else max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / s) if a.size else 0.0
