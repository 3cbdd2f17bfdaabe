"""The oracle restatement (oracle/dmph_oracle.c) against the golden fixtures
that the reference solver itself produced (tests/golden/make_golden.py)."""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from helpers import GOLD, GOLDEN, fingerprint_ok, load_scene
from oracle.oracle import Oracle
from dem_mph_b200 import generator


def test_generator_reproduces_shipped_grid():
    """Known-answer test: results/SYSU/2mm/DEM.boid -> DEM.grid byte for byte."""
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "DEM.grid")
        n = generator.boid_to_grid(os.path.join(GOLDEN, "sysu2mm", "DEM.boid"), out)
        assert n == 19913
        with open(out, "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == GOLD["generator_kat"]["sysu2mm"]


@pytest.mark.parametrize("name", ["shapes", "errors"])
def test_generator_shapes_match_reference_generator(name):
    """Every block shape the reference generator reads (Cuboid, Cuboid2,
    Cyboid, Cyboid2, Recboid, Recboid2), and its handling of an unknown shape
    and of a block with a field its reader rejects: the .grid is byte for
    byte the one the reference generator wrote for the same .boid (SHA-256
    recorded by tests/golden/make_generator_golden.py)."""
    import warnings
    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, name + ".grid")
        with warnings.catch_warnings(record=True) as caught:
            warnings.simplefilter("always")
            generator.boid_to_grid(os.path.join(GOLDEN, "shapes", name + ".boid"), out)
        with open(out, "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == GOLD["generator_kat"]["shapes/" + name]
    assert bool(caught) == (name == "errors")


@pytest.mark.parametrize("name", sorted(GOLD["scenes"]))
def test_oracle_matches_reference(name):
    rec = GOLD["scenes"][name]
    p, typ, x, v = load_scene(name)
    o = Oracle(p, typ, x, v)
    done = 0
    for s in sorted(int(k) for k in rec["steps"]):
        o.step(s - done)
        done = s
        gold = rec["steps"][str(s)]
        bad = []
        for arr, fp in gold["arrays"].items():
            ok, msg = fingerprint_ok(o.get(arr), fp)
            if not ok:
                bad.append("%s: %s" % (arr, msg))
        assert not bad, "step %d: %s" % (s, "; ".join(bad))
        meta = gold["meta"]
        assert o.scalar("N0a") == meta["N0a"] and o.scalar("N0p") == meta["N0p"]
        assert o.scalar("Rebuilds") == meta["Rebuilds"]
        assert o.scalar("Time") == meta["Time"]
        assert [o.scalar("CellCount%d" % d) for d in range(3)] == meta["CellCount"]


@pytest.mark.parametrize("name", ["small3d", "sysu2mm"])
def test_oracle_cell_sort_alone_matches_full_oracle(name):
    """dmph_oracle_cell_sort (the checker of the library's allocation-free
    sort) gives the CellIndex and ParticleIndex of the full oracle's first
    sort, which the golden fixtures pin to the reference."""
    from oracle import oracle as orc
    p, typ, x, v = load_scene(name)
    o = Oracle(p, typ, x, v)
    key, perm = orc.cell_sort(p, typ, x)
    assert np.array_equal(key, o.get("CellIndex")[:len(typ)])
    assert np.array_equal(perm, o.get("ParticleIndex"))
