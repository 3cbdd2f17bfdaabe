"""Generate the golden fixtures under tests/golden/ from the REFERENCE itself.

Run where the reference tree is present ($DMPH_REFERENCE_DIR, default a
`reference` checkout beside this repository) and oracle/_ref is built
(make -C oracle ref):

    python tests/golden/make_golden.py [--ref <reference tree>]

It copies the two shipped SYSU case descriptions (dem.data and DEM.boid,
results/SYSU/{2mm,0.8mm}) as small input fixtures, records the SHA-256 of the
shipped results/SYSU/2mm/DEM.grid (the generator known-answer test), and runs
the reference solver harness oracle/_ref/ref_dump{2d,3d} on four scenes.  For
every dumped array it stores a fingerprint: the SHA-256 of integer arrays and
three checksums of floating-point arrays (sum, sum of |x| and an
index-weighted sum), which pin the arrays to ~1e-12 without committing them.
"""
import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dem_mph_b200 import files, generator, scenes  # noqa: E402
from oracle.oracle import read_ref_dump, REF_DIR  # noqa: E402

SCENES = {
    # name: (kind, steps to dump)
    "sysu2mm": ("2d", [0, 1, 2, 50]),
    "sysu08mm": ("2d", [0, 2]),
    "small3d": ("3d", [0, 1, 150]),
    "small3d_st": ("3d", [0, 1, 30]),
}


def fingerprint(a):
    a = np.asarray(a)
    if a.dtype.kind in "iu":
        return {"dtype": str(a.dtype), "n": int(a.size), "sha256": hashlib.sha256(a.tobytes()).hexdigest()}
    f = a.astype(np.float64).ravel()
    w = (np.arange(f.size) % 97 + 1).astype(np.float64)
    return {"dtype": str(a.dtype), "n": int(a.size), "sum": float(np.sum(f)), "abs": float(np.sum(np.abs(f))),
            "wsum": float(np.sum(f * w)), "nan": int(np.sum(np.isnan(f)))}


def small3d_st_params(p):
    """small3d with the surface-tension model switched on (non-zero
    InteractionRatio and SurfaceTension), to cover those code paths."""
    q = p.copy()
    q.surface_tension[1] = 0.072
    q.surface_tension[2] = 0.03
    for a, b, r in ((1, 1, 1.0), (1, 2, 0.4), (2, 1, 0.6), (1, 4, 0.2), (4, 1, 0.3), (2, 2, 0.5)):
        q.interaction_ratio[a][b] = r
    return q


def scene_inputs(name, workdir, ref):
    """Write dem.data + grid for a scene into workdir; returns (data, grid)."""
    data = os.path.join(workdir, "dem.data")
    grid = os.path.join(workdir, "scene.grid")
    if name.startswith("sysu"):
        case = "2mm" if name == "sysu2mm" else "0.8mm"
        src = os.path.join(ref, "results", "SYSU", case)
        shutil.copyfile(os.path.join(src, "dem.data"), data)
        generator.boid_to_grid(os.path.join(src, "DEM.boid"), grid)
    else:
        s = scenes.small()
        p = s.params if name == "small3d" else small3d_st_params(s.params)
        files.write_data_file(data, p)
        files.write_grid(grid, p, s.type, s.x, s.v)
    return data, grid


def main():
    ap = argparse.ArgumentParser()
    default_ref = os.environ.get("DMPH_REFERENCE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))), "reference")
    ap.add_argument("--ref", default=default_ref)
    args = ap.parse_args()
    out = {"generator_kat": {}, "scenes": {}}
    # input fixtures
    for case, tag in (("2mm", "sysu2mm"), ("0.8mm", "sysu08mm")):
        d = os.path.join(HERE, tag)
        os.makedirs(d, exist_ok=True)
        for fn in ("dem.data", "DEM.boid"):
            shutil.copyfile(os.path.join(args.ref, "results", "SYSU", case, fn), os.path.join(d, fn))
    with open(os.path.join(args.ref, "results", "SYSU", "2mm", "DEM.grid"), "rb") as f:
        out["generator_kat"]["sysu2mm"] = hashlib.sha256(f.read()).hexdigest()
    # reference dumps
    for name, (kind, steps) in SCENES.items():
        with tempfile.TemporaryDirectory() as tmp:
            data, grid = scene_inputs(name, tmp, args.ref)
            exe = os.path.join(REF_DIR, "ref_dump2d" if kind == "2d" else "ref_dump3d")
            dump = os.path.join(tmp, "out")
            cmd = [exe, data, grid, dump, str(max(steps))] + [str(s) for s in steps if s > 0]
            subprocess.run(cmd, check=True, capture_output=True)
            rec = {"dim": 2 if kind == "2d" else 3, "steps": {}}
            for s in steps:
                d = read_ref_dump(os.path.join(dump, "step%d" % s))
                meta = d.pop("meta")
                rec["steps"][str(s)] = {"arrays": {k: fingerprint(v) for k, v in sorted(d.items())},
                                        "meta": meta}
            with open(grid, "rb") as f:
                rec["grid_sha256"] = hashlib.sha256(f.read()).hexdigest()
            out["scenes"][name] = rec
            print(name, "done", file=sys.stderr)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
