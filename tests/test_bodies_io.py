"""Rigid bodies at the drop-in boundary, host side (no GPU): the body sidecar
file through the C ABI, its error handling, and the bodies found by contact
at 1.01 dx, which must be the seeded generator's own bodies on the benchmark
scenes (the reference's .grid carries no body, generator/generator.cpp:97,
211-214, so one of the two is needed to run bodies from files)."""
import os
import tempfile

import numpy as np
import pytest

from dem_mph_b200 import scenes, solver


def canon(body):
    """body ids relabelled by first occurrence (-1 kept)"""
    out = np.full(len(body), -1, np.int64)
    seen = {}
    for i, b in enumerate(body):
        if b >= 0:
            out[i] = seen.setdefault(int(b), len(seen))
    return out


def test_sidecar_roundtrip():
    s = scenes.small()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "DEM.bodies")
        solver.write_bodies(path, s.body, s.body_density)
        b, rho = solver.read_bodies(path)
    assert np.array_equal(b, s.body) and np.array_equal(rho, s.body_density)


@pytest.mark.parametrize("text,why", [("DMPH_BODIES 2\n0 0\n", "version"),
                                      ("DMPH_BODIES 1\n1 2\n500\n0\n1\n", "row body out of range"),
                                      ("DMPH_BODIES 1\n1 1\n-3\n0\n", "negative density"),
                                      ("DMPH_BODIES 1\n2 1\n500\n", "truncated")])
def test_sidecar_errors(text, why):
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "bad.bodies")
        with open(path, "w") as f:
            f.write(text)
        with pytest.raises(solver.DmphError) as e:
            solver.read_bodies(path)
    assert e.value.code in (-4, -7), why


@pytest.mark.parametrize("name", ["small", "config1", "config2"])
def test_bodies_by_contact_are_the_generator_bodies(name):
    s = {"small": scenes.small, "config1": scenes.config1, "config2": scenes.config2}[name]()
    b, rho = solver.bodies_from_contacts(s.params, s.type, s.x)
    assert len(rho) == len(s.body_density)
    assert np.array_equal(canon(b), canon(s.body))
    solid = (s.type >= 2) & (s.type < 4)
    assert np.all(b[solid] >= 0) and np.all(b[~solid] == -1)
    # each body's density is its first row's type density
    rows = np.flatnonzero(b >= 0)
    ids, first = np.unique(b[rows], return_index=True)
    assert np.array_equal(ids, np.arange(len(rho)))
    assert np.array_equal(rho, np.array(list(s.params.density))[s.type[rows[first]]])


def test_touching_blocks_join():
    """two debris particles at exactly dx (and at 1.005 dx) are one body,
    at 1.02 dx two; across the periodic boundary too"""
    s = scenes.small()
    p = s.params
    dx = p.particle_spacing
    lo = np.array(p.domain_min)
    W = np.array(p.domain_max) - lo
    x = np.array([[lo[0] + 0.5 * dx, lo[1] + 0.5, lo[2] + 0.2],
                  [lo[0] + W[0] - 0.505 * dx, lo[1] + 0.5, lo[2] + 0.2],   # 1.005 dx across the boundary
                  [lo[0] + 0.3, lo[1] + 0.5, lo[2] + 0.2],
                  [lo[0] + 0.3 + 1.02 * dx, lo[1] + 0.5, lo[2] + 0.2]])
    typ = np.array([2, 2, 2, 3], np.int32)
    b, rho = solver.bodies_from_contacts(p, typ, x)
    assert list(b) == [0, 0, 1, 2] and len(rho) == 3
    assert rho[2] == p.density[3]
