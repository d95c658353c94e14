"""Crossing-walk cases of popup/src/obstacles/tests/crossings.rs, re-encoded on this library's
lattice scenes, run against the oracle's restatement of the walk."""

import numpy as np

from helpers import Stock, square
from oracle import oracle


def crossings_of(stock, frm, to):
    scene = oracle.OracleScene(stock.scene())
    return scene.crossings(stock.steps(frm), stock.steps(to))


def test_tangent_contact_keeps_roof_and_containment_parity():
    # crossings.rs:6-36
    for coincident in (False, True):
        stock = Stock()
        stock.building(1, 6.0, [square(0.0, 0.0, 5.0)])
        stock.building(2, 9.0, [[(100.0, 0.0), (110.0, 10.0), (100.0, 20.0), (90.0, 10.0)]])
        centre = 120.0 if coincident else 200.0
        stock.building(2, 9.0, [square(centre, 0.0, 20.0)])
        scene = oracle.OracleScene(stock.scene())
        assert scene.enclosing(stock.steps((0.0, 0.0)))[0] == 1
        c = scene.crossings(stock.steps((0.0, 0.0)), stock.steps((300.0, 0.0)))
        assert len(c["t"]) == (3 if coincident else 4)
        other = c["bounds_roof"][c["footprint"] == 2]
        assert bool(other[0]) == coincident
        assert other[1:].all()


def test_ray_through_square_crosses_twice():
    stock = Stock()
    stock.building(7, 12.0, [square(500.0, 0.0, 10.0)])
    c = crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))
    assert len(c["t"]) == 2 and c["t"][0] < c["t"][1]
    assert abs(c["t"][0] - 0.49) < 0.005 and abs(c["t"][1] - 0.51) < 0.005
    assert (c["footprint"] == 7).all() and c["building"].all()


def test_ray_beside_square_misses():
    stock = Stock()
    stock.building(1, 12.0, [square(500.0, 100.0, 10.0)])
    assert len(crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))["t"]) == 0


def test_receiver_inside_footprint_sees_entry_only():
    stock = Stock()
    stock.building(3, 20.0, [square(1000.0, 0.0, 15.0)])
    c = crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))
    assert len(c["t"]) == 1 and 0.0 < c["t"][0] < 1.0


def test_long_wall_crossing_reported_once():
    stock = Stock()
    stock.wall(9, 4.0, [(500.0, -400.0), (500.0, 400.0)])
    c = crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))
    assert len(c["t"]) == 1 and not c["building"][0] and abs(c["t"][0] - 0.5) < 0.005


def test_two_buildings_sorted_by_chainage():
    stock = Stock()
    stock.building(1, 6.0, [square(300.0, 0.0, 10.0)])
    stock.building(2, 9.0, [square(700.0, 0.0, 10.0)])
    c = crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))
    assert list(c["footprint"]) == [1, 1, 2, 2]
    assert np.all(np.diff(c["t"]) > 0)


def test_diagonal_ray_hits_offset_wall_once():
    stock = Stock()
    stock.wall(4, 5.0, [(400.0, 260.0), (640.0, 100.0)])
    assert len(crossings_of(stock, (0.0, 0.0), (1000.0, 500.0))["t"]) == 1


def test_shallow_wall_with_many_intervening_hits_reported_once():
    stock = Stock()
    stock.wall(99, 4.0, [(100.0, -40.0), (2000.0, 80.0)])
    for i in range(10):
        stock.building(i + 1, 6.0, [square(500.0 + 120.0 * i, 0.0, 8.0)])
    c = crossings_of(stock, (0.0, 0.0), (2000.0, 0.0))
    assert (c["footprint"] == 99).sum() == 1
    assert len(c["t"]) == 21


def test_ring_vertex_hit_is_single_candidate():
    stock = Stock()
    stock.building(5, 10.0, [square(500.0, 100.0, 100.0)])
    corner = np.array([400.0, 0.0])
    c = crossings_of(stock, corner - 100.0, corner + 300.0)
    assert (np.abs(c["t"] - 0.25) < 0.01).sum() <= 1
    assert len(c["t"]) > 0


def test_vertical_ray_crosses_horizontal_wall():
    stock = Stock()
    stock.wall(1, 3.0, [(-50.0, 300.0), (50.0, 300.0)])
    c = crossings_of(stock, (0.0, 0.0), (0.0, 600.0))
    assert len(c["t"]) == 1 and abs(c["t"][0] - 0.5) < 0.005


def test_ray_from_far_outside_still_hits():
    stock = Stock()
    stock.building(2, 9.0, [square(0.0, 0.0, 20.0)])
    assert len(crossings_of(stock, (-5000.0, 0.0), (5000.0, 0.0))["t"]) == 2


def test_reversed_ray_is_symmetric():
    stock = Stock()
    stock.building(1, 6.0, [square(300.0, 0.0, 10.0)])
    f = crossings_of(stock, (0.0, 0.0), (1000.0, 0.0))
    r = crossings_of(stock, (1000.0, 0.0), (0.0, 0.0))
    np.testing.assert_allclose(np.sort(f["t"]), np.sort(1.0 - r["t"]), atol=1e-12)
