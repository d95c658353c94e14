"""The oracle's crossing walk and terrain profile with ends off the integer lattice, as the
reference's walk takes a line node's ray (popup/src/obstacles/mod.rs:61-73): on lattice ends they
read as the integer forms bit for bit, and on any ends the walk's list is the list of every edge
against the ray with the same deduplication (the reference's own check of its walk,
popup/src/obstacles/tests/mod.rs:198-229, crossings.rs:186-200)."""

import numpy as np
import pytest

from helpers import Stock, square
from oracle import oracle
from quietmap_b200 import scenes


@pytest.fixture(scope="module", params=["road", "terrain"])
def scene(request):
    if request.param == "road":
        return scenes.road_square()[0]
    return scenes.terrain_square(scale=0.125)[0]


def _same(a, b):
    for key in ("t", "footprint", "edge", "bounds_roof", "building"):
        np.testing.assert_array_equal(a[key], b[key])


def test_lattice_ends_read_as_the_integer_walk(scene):
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(23)
    ext = np.array(scene.extent_steps)
    for _ in range(400):
        a, b = rng.integers(0, ext, 2), rng.integers(0, ext, 2)
        _same(ora.crossings_f64(a.astype(np.float64), b.astype(np.float64)), ora.crossings(a, b))
        h, t, z, g = ora.profile_f64(a.astype(np.float64), b.astype(np.float64))
        h0, t0, z0, g0 = ora.profile(a, b)
        assert h == h0
        np.testing.assert_array_equal(t, t0)
        np.testing.assert_array_equal(z, z0)
        np.testing.assert_array_equal(g, g0)


def test_off_lattice_ends_find_every_crossing(scene):
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(29)
    ext = np.array(scene.extent_steps, dtype=np.float64)
    for _ in range(1500):
        a, b = rng.uniform(0.0, 1.0, 2) * ext, rng.uniform(0.0, 1.0, 2) * ext
        _same(ora.crossings_f64(a, b), ora.crossings_every(a, b))


def test_a_vertical_ray_past_two_footprints_off_the_lattice():
    """crossings.rs:186-200, the ray shifted by a third of a step off the lattice."""
    stock = Stock()
    stock.building(0, 10.0, [square(0.0, 0.0, 10.0)])
    stock.building(1, 10.0, [square(0.0, 200.0, 10.0)])
    ora = oracle.OracleScene(stock.scene())
    frm = stock.steps((0.0, 2_000.0)).astype(np.float64) + [1.0 / 3.0, 0.0]
    to = stock.steps((0.0, -2_000.0)).astype(np.float64) + [1.0 / 3.0, 0.0]
    walked = ora.crossings_f64(frm, to)
    assert len(walked["t"]) == 4
    _same(walked, ora.crossings_every(frm, to))
