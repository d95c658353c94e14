"""The receiver skyline of the line quadrature (popup/src/obstacles/skyline.rs) restated in the
oracle, pinned to the reference's own tests (popup/src/obstacles/tests/skyline.rs): in-range
edges and their bearings, a box under the sight line pruned whole, a low wall pruned on its own
height, a multi-cell wall repeating one arc, a wall half a metre away kept and one through the
receiver dropped."""

import math

from oracle import obstacles as ob

STEP_M = 0.1919                      # a step at 50 N (the reference's stock origin), metres
ORIGIN = (2212 * 32768 + 12345, 1387 * 32768 + 23456)  # the receiver, exactly on a step
EAST = (-0.5, 0.5)


class Stock:
    """Outlines on the global step lattice around the receiver: metres east and north rounded to
    the nearest step (y grows south)."""

    def __init__(self):
        self.outlines = []

    def steps(self, p):
        return (ORIGIN[0] + round(p[0] / STEP_M), ORIGIN[1] - round(p[1] / STEP_M))

    def building(self, fp, height, ring):
        vertices = [self.steps(p) for p in ring]
        self.outlines.append(dict(footprint_id=fp, kind=ob.EXTERIOR, height_m=height, vertices=vertices + vertices[:1]))

    def wall(self, fp, height, points):
        self.outlines.append(dict(footprint_id=fp, kind=ob.WALL, height_m=height,
                                  vertices=[self.steps(p) for p in points]))

    def arcs(self, wedge, radius_m, los_floor_m):
        return ob.Skyline(self.outlines, (STEP_M, STEP_M)).arcs(ORIGIN, wedge[0], wedge[1], radius_m, los_floor_m)


def square(east, north, half):
    return [(east - half, north - half), (east + half, north - half), (east + half, north + half),
            (east - half, north + half)]


def distinct(arcs):
    """An edge listed in several cells is handed over once per cell."""
    out = []
    for a in sorted(arcs, key=lambda a: (a[0], a[1])):
        if not out or out[-1] != a:
            out.append(a)
    return out


def test_skyline_reports_in_range_edges_with_their_bearing():
    stock = Stock()
    stock.building(0, 8.0, square(200.0, 0.0, 15.0))
    stock.building(1, 8.0, square(2000.0, 0.0, 15.0))
    found = distinct(stock.arcs(EAST, 500.0, 0.0))
    assert len(found) == 4, found
    for lo, hi, nearest in found:
        assert hi - lo < math.pi
        assert abs(lo) < 0.2 and abs(hi) < 0.2
        assert 184.8 <= nearest <= 216.2
    assert stock.arcs(EAST, 100.0, 0.0) == []
    assert stock.arcs((2.0, 2.5), 500.0, 0.0) == []


def test_a_box_under_the_sight_line_is_pruned_whole():
    for height, expected in ((8.0, 4), (4.0, 0), (3.0, 0)):
        stock = Stock()
        stock.building(0, height, square(200.0, 0.0, 15.0))
        assert len(distinct(stock.arcs(EAST, 500.0, 4.0))) == expected, height


def test_a_low_wall_is_pruned_on_its_own_height_not_its_cells():
    stock = Stock()
    stock.building(0, 20.0, square(200.0, 0.0, 20.0))
    stock.wall(1, 3.0, [(190.0, 0.0), (210.0, 0.0)])
    wall = lambda arc: abs(arc[2] - 190.0) < 0.5
    at_ground = stock.arcs(EAST, 500.0, 0.0)
    assert any(wall(a) for a in at_ground)
    assert len(distinct(at_ground)) == 5
    above = stock.arcs(EAST, 500.0, 4.0)
    assert not any(wall(a) for a in above)
    assert len(distinct(above)) == 4


def test_a_multicell_wall_repeats_one_arc():
    stock = Stock()
    stock.wall(0, 8.0, [(60.0, -400.0), (60.0, 400.0)])
    found = stock.arcs((-1.5, 1.5), 1000.0, 0.0)
    assert len(found) > 1
    assert all(a[0] == found[0][0] and a[1] == found[0][1] for a in found)
    assert found[0][0] < -1.0 and found[0][1] > 1.0


def test_a_wall_half_a_metre_away_is_kept_and_one_through_the_receiver_is_not():
    stock = Stock()
    stock.wall(0, 3.0, [(0.5, -5.0), (0.5, 5.0)])
    stock.wall(1, 3.0, [(-5.0, 0.0), (5.0, 0.0)])
    found = distinct(stock.arcs(EAST, 50.0, 0.0))
    assert len(found) == 1, found
    assert abs(found[0][2] - 0.5) < 0.2


def _scene_and_restated(seed):
    """A random stock scene of buildings and walls, and the same outlines for the restated
    skyline: steps with y negated (the reference's lattice grows south), heights as the scene
    holds them (float32)."""
    import numpy as np

    from helpers import Stock as SceneStock

    rng = np.random.default_rng(seed)
    stock = SceneStock()
    for fp in range(1, 41):
        cx, cy = rng.uniform(-150.0, 150.0, 2)
        if rng.random() < 0.7:
            half = rng.uniform(2.0, 15.0)
            stock.building(fp, float(rng.uniform(1.0, 25.0)), [[(cx - half, cy - half), (cx + half, cy - half),
                                                                (cx + half, cy + half), (cx - half, cy + half)]])
        else:
            points = [(cx, cy)] + [tuple(rng.uniform(-150.0, 150.0, 2)) for _ in range(int(rng.integers(1, 4)))]
            stock.wall(fp, float(rng.uniform(0.5, 6.0)), points)
    outlines = []
    for verts, (first, count, fp, height, building) in zip(stock.verts, stock.records):
        outlines.append(dict(footprint_id=fp, kind=ob.EXTERIOR if building else ob.WALL,
                             height_m=float(np.float32(height)), vertices=[(int(x), -int(y)) for x, y in verts]))
    return stock, ob.Skyline(outlines, (stock.step_m, stock.step_m))


def test_the_oracle_scene_skyline_is_the_restated_one():
    """The C++ skyline over a scene hands over the same arcs, in the same order and to the bit,
    as the restatement pinned above, across receivers, wedges (some wrapping past pi), radii and
    sight-line floors that prune walls and whole cells."""
    import numpy as np

    from oracle import oracle

    stock, restated = _scene_and_restated(11)
    ora = oracle.OracleScene(stock.scene())
    rng = np.random.default_rng(5)
    total = 0
    for _ in range(60):
        r = stock.steps(rng.uniform(-120.0, 120.0, 2))
        lo = rng.uniform(-math.pi, math.pi)
        hi = lo + rng.uniform(0.01, 3.0)
        radius, floor = rng.uniform(5.0, 250.0), float(rng.choice([0.0, 0.05, 3.0, 12.0]))
        got = ora.skyline_arcs(r, lo, hi, radius, floor)
        want = np.array(restated.arcs((int(r[0]), -int(r[1])), lo, hi, radius, floor)).reshape(-1, 3)
        assert np.array_equal(got, want), (r, lo, hi, radius, floor, len(got), len(want))
        total += len(got)
    assert total > 500
