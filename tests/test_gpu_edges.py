"""Edge cases through the C ABI: empty inputs, silent spectra, NaN and out-of-range levels, a
one-receiver grid, a receiver inside a building, flights with no segments."""

import numpy as np
import pytest

from helpers import Stock, point_sources, square
from oracle import oracle
from quietmap_b200 import native, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return native.Context(0)


def test_empty_inputs(ctx):
    assert ctx.zwicker(np.zeros((0, 28), np.float32)).shape == (0,)
    assert np.all(ctx.level_histogram(np.zeros(0, np.float32)) == 0)
    scene, full = scenes.road_square()
    dev = ctx.scene(scene)
    counts, _, _, _, status = dev.list_crossings(np.zeros((0, 2)), np.zeros((0, 2)))
    assert counts.shape == (0,) and status.shape == (0,)


def test_silent_spectra_and_odd_levels(ctx):
    silent = np.full((3, 28), -np.inf, np.float32)
    assert np.all(ctx.zwicker(silent) == 0.0)
    assert np.allclose(ctx.zwicker(silent), oracle.zwicker_many(silent.astype(np.float64)))
    levels = np.array([np.nan, -np.inf, np.inf, -1e9, 1e9, -30.0, -29.95, 149.9, 150.0], np.float32)
    counts = ctx.level_histogram(levels, -30.0, 0.1, 1800)
    ref = oracle.level_histogram(levels.astype(np.float64), -30.0, 0.1, 1800)
    assert np.array_equal(counts, ref)
    assert counts.sum() == len(levels)


def test_one_receiver_grid_and_a_receiver_inside_a_building(ctx):
    stock = Stock(side_m=400.0, offset_m=200.0)
    stock.building(5, 10.0, [square(0.0, 0.0, 8.0)])
    stock.building(6, 6.0, [square(40.0, 10.0, 5.0)])
    scene = stock.scene(sources=point_sources(stock, [(-80.0, 3.0), (90.0, -20.0), (10.0, 60.0)]))
    dev = ctx.scene(scene)
    ora = oracle.OracleScene(scene)
    for xy in [(1.0, 2.0), (60.0, 30.0)]:  # inside building 5, then outside both
        o = stock.steps(xy)
        grid = scenes.Grid(origin=(int(o[0]), int(o[1])), spacing=32, nx=1, ny=1)
        bands, dba, lden, hist, st = dev.paint_grid(grid)
        e, l, _ = ora.paint_grid(grid)
        assert st["paths"] == 3
        np.testing.assert_allclose(bands[0], 10 * np.log10(e[0]), atol=0.05)
        np.testing.assert_allclose(lden[0], 10 * np.log10(l[0]), atol=0.05)
        assert hist.sum() == 1


def test_flights_without_segments_are_silent(ctx):
    f = scenes.flights_square(n_flights=1, receivers=8)
    f.segments = f.segments[:0]
    lae, thirds, sone = ctx.flight_grid(f)
    assert np.all(np.isneginf(lae)) and np.all(np.isneginf(thirds)) and np.all(sone == 0.0)
