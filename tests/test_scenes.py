"""Seeded benchmark scenes (dem_mph_b200.scenes) that only their sizes pin:
config 5, the surrogate's production case (3.2 x 1.0 x 1.0 m tank at
3.5 mm, ~4 M fluid, 1000 debris cuboids)."""
import numpy as np

from dem_mph_b200 import scenes


def test_config5_sizes_and_bodies():
    s = scenes.config5()
    c = s.counts
    c = c() if callable(c) else c
    assert 3.9e6 <= c["fluid"] <= 4.2e6, c
    assert len(s.body_density) == 1000
    assert np.all((s.body_density >= 400.0) & (s.body_density <= 900.0))
    solid = (s.type >= 2) & (s.type < 4)
    assert np.array_equal(np.unique(s.body[solid]), np.arange(1000)) and np.all(s.body[~solid] == -1)
    sizes = np.bincount(s.body[solid])
    assert sizes.min() >= 27 and sizes.max() <= 216  # cuboids of 3-6 particles a side
    # the debris sit on the floor downstream of the column, inside the tank
    xs = s.x[solid]
    assert xs[:, 0].min() > 0.5 and xs[:, 0].max() < 3.2 and xs[:, 1].min() >= 0.0
    assert xs[:, 2].min() > 0.0 and xs[:, 2].max() < 1.0
    # same seed, same scene
    t = scenes.config5()
    assert np.array_equal(s.x, t.x) and np.array_equal(s.body, t.body)
