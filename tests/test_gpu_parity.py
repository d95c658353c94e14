"""Parity of the CUDA painter with the FP64 oracle, through the C ABI, on seeded scenes.

Bars: crossing lists bit-exact (edge ids, chainage t, flags); histogram counts bit-exact given the
device's own cell levels; cell band levels, dBA and Lden within 0.05 dB of the oracle; Zwicker
within 0.5 %; per-pair energies within 0.05 dB at the maximum.
"""

import numpy as np
import pytest

from helpers import Stock, square
from oracle import oracle
from quietmap_b200 import native, scenes

pytestmark = pytest.mark.gpu

TOL_DB = 0.05


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def road():
    return scenes.road_square()


@pytest.fixture(scope="module")
def terrain():
    return scenes.terrain_square(scale=0.125)


def _rays(scene, rng, n):
    ext = np.array(scene.extent_steps)
    frm = rng.integers(0, ext, (n, 2))
    to = rng.integers(0, ext, (n, 2))
    # Half of them from real source points to receivers.
    k = n // 2
    idx = rng.integers(0, len(scene.sources), k)
    frm[:k, 0] = scene.sources["x"][idx]
    frm[:k, 1] = scene.sources["y"][idx]
    return frm, to


def _assert_crossings_equal(dev_scene, ora, frm, to):
    counts, edges, t, flags, status = dev_scene.list_crossings(frm, to)
    assert not status.any()
    for i in range(len(frm)):
        ref = ora.crossings(frm[i], to[i])
        n = len(ref["t"])
        assert counts[i] == n, (i, counts[i], n)
        np.testing.assert_array_equal(edges[i, :n], ref["edge"])
        np.testing.assert_array_equal(t[i, :n], ref["t"])  # bit for bit
        np.testing.assert_array_equal(flags[i, :n] & 1, ref["building"].astype(np.uint32))
        np.testing.assert_array_equal((flags[i, :n] >> 1) & 1, ref["bounds_roof"].astype(np.uint32))


def test_crossing_lists_are_bit_exact_on_the_road_square(ctx, road):
    scene, _ = road
    dev, ora = ctx.scene(scene), oracle.OracleScene(scene)
    frm, to = _rays(scene, np.random.default_rng(5), 3000)
    _assert_crossings_equal(dev, ora, frm, to)


def test_crossing_lists_are_bit_exact_on_the_terrain_square(ctx, terrain):
    scene, _ = terrain
    dev, ora = ctx.scene(scene), oracle.OracleScene(scene)
    frm, to = _rays(scene, np.random.default_rng(6), 3000)
    _assert_crossings_equal(dev, ora, frm, to)


def test_crossing_edge_cases_corners_tangents_and_walls(ctx):
    stock = Stock()
    stock.building(1, 6.0, [square(0.0, 0.0, 5.0)])
    stock.building(2, 9.0, [[(100.0, 0.0), (110.0, 10.0), (100.0, 20.0), (90.0, 10.0)]])
    stock.building(2, 9.0, [square(120.0, 0.0, 20.0)])
    stock.building(5, 10.0, [square(500.0, 100.0, 100.0)])
    stock.wall(9, 4.0, [(500.0, -400.0), (500.0, 400.0)])
    stock.wall(99, 4.0, [(100.0, -40.0), (2000.0, 80.0)])
    scene = stock.scene()
    dev, ora = ctx.scene(scene), oracle.OracleScene(scene)
    rays = [((0.0, 0.0), (300.0, 0.0)), ((300.0, -100.0), (700.0, 300.0)), ((0.0, 0.0), (2000.0, 0.0)),
            ((400.0, 0.0), (400.0, 300.0)), ((-100.0, 10.0), (300.0, 10.0)), ((90.0, -50.0), (90.0, 50.0)),
            ((0.0, 0.0), (0.0, 0.0))]
    frm = np.array([stock.steps(a) for a, _ in rays])
    to = np.array([stock.steps(b) for _, b in rays])
    _assert_crossings_equal(dev, ora, frm, to)


def test_the_painters_warp_crossing_walk_lists_what_single_rays_list(ctx, terrain):
    """The grid painter lists the crossings of a warp's 32 rays together (a sweep over the union of
    their cells, staged in shared memory); every ray must get exactly the crossings the single-ray
    walk of qm_list_crossings gives it. Checked by the total over a tile's receivers and 4,000
    sources in every direction, the receivers standing outside every building (the single-ray entry
    keeps a receiver's own walls)."""
    scene, grid = terrain
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(13)
    ext = np.array(scene.extent_steps)
    for _ in range(200):
        o = rng.integers(0, ext - 16 * grid.spacing)
        g = scenes.Grid(origin=(int(o[0]), int(o[1])), spacing=grid.spacing, nx=16, ny=8, source_begin=0,
                        source_end=4000)
        rxy = g.receiver_xy()
        if not ora.enclosing(rxy).any():
            break
    dev = ctx.scene(scene)
    _, _, _, _, stats = dev.paint_grid(g)
    assert stats["failed_paths"] == 0
    src = np.stack([scene.sources["x"][:4000], scene.sources["y"][:4000]], axis=1)
    frm = np.repeat(src, len(rxy), axis=0)
    to = np.tile(rxy, (len(src), 1))
    counts, _, _, _, status = dev.list_crossings(frm, to)
    assert not status.any()
    assert stats["crossings"] == int(counts.sum()), (stats["crossings"], int(counts.sum()))


def _levels_db(energy):
    with np.errstate(divide="ignore"):
        return 10.0 * np.log10(energy)


def _check_grid(ctx, scene, grid, sample_cells, rng):
    dev = ctx.scene(scene)
    bands, dba, lden, hist, stats = dev.paint_grid(grid)
    assert stats["paths"] == grid.cells * len(scene.sources)
    # Paths over the per-path capacities are re-run on the device; they stay rare.
    assert stats["failed_paths"] <= stats["paths"] // 1000
    # Histogram: exact counts of the device's own dBA levels under the reference's bin rule.
    ref_hist = oracle.level_histogram(dba.astype(np.float64), grid.level_min_db, grid.bin_db, grid.n_bins)
    np.testing.assert_array_equal(hist, ref_hist)
    # Cell levels against the oracle on a seeded sample of cells.
    ora = oracle.OracleScene(scene)
    cells = np.sort(rng.choice(grid.cells, sample_cells, replace=False))
    worst = 0.0
    for c in cells:
        e, l, _ = ora.paint_grid(grid, int(c), int(c) + 1)
        ref_bands = _levels_db(e[0])
        ref_dba = _levels_db(e[0].sum())
        ref_lden = _levels_db(l[0])
        ok = np.isfinite(ref_bands) & (ref_bands > ref_dba - 60.0)
        err = np.abs(bands[c][ok] - ref_bands[ok])
        worst = max(worst, float(err.max(initial=0.0)), abs(dba[c] - ref_dba), abs(lden[c] - ref_lden))
        assert err.max(initial=0.0) < TOL_DB, (c, bands[c], ref_bands)
        assert abs(dba[c] - ref_dba) < TOL_DB, (c, dba[c], ref_dba)
        assert abs(lden[c] - ref_lden) < TOL_DB, (c, lden[c], ref_lden)
    return worst


def test_road_square_cells_match_the_oracle(ctx, road):
    scene, grid = road
    _check_grid(ctx, scene, grid, 24, np.random.default_rng(7))


def test_terrain_square_cells_match_the_oracle(ctx, terrain):
    scene, grid = terrain
    # A 32 x 32 block of receivers over the scaled terrain square, every source.
    sub = scenes.Grid(origin=grid.origin, spacing=grid.spacing * 8, nx=32, ny=32)
    _check_grid(ctx, scene, sub, 12, np.random.default_rng(8))


def _pair_case(scene, rng, n_receivers, n_pairs):
    ext = np.array(scene.extent_steps)
    rxy_steps = rng.integers(1, ext - 1, (n_receivers, 2))
    rxy_m = rxy_steps * scene.step_m
    sop = rng.integers(0, len(scene.sources), n_pairs).astype(np.uint32)
    rop = np.sort(rng.integers(0, n_receivers, n_pairs)).astype(np.uint32)
    return rxy_steps, rxy_m, sop, rop


def _check_pairs(ctx, scene, rng):
    dev, ora = ctx.scene(scene), oracle.OracleScene(scene)
    n_receivers, n_pairs = 64, 4000
    rxy_steps, rxy_m, sop, rop = _pair_case(scene, rng, n_receivers, n_pairs)
    own = ora.enclosing(rxy_steps)
    point = np.arange(n_receivers, dtype=np.uint32)
    weight = rng.uniform(0.5, 2.0, n_pairs)
    sums, bands, status, points = dev.evaluate_pairs(rxy_m, np.full(n_receivers, 4.0), own, point, sop, rop,
                                                     weight.astype(np.float32), n_receivers)
    assert not status.any()
    # Oracle receivers: altitude = ground + 4 m (the ground is the same bilinear rule).
    ground = np.array([ora.profile(p, p)[2][0] for p in rxy_steps])
    ref_sums, ref_bands, ref_points = ora.evaluate_pairs(rxy_steps, ground + 4.0, own, point, sop, rop, weight,
                                                         n_receivers)
    got, ref = _levels_db(sums.astype(np.float64)), _levels_db(ref_sums)
    # Silent sums (no energy in a state or period) must be silent on both sides.
    assert np.array_equal(np.isfinite(got), np.isfinite(ref))
    heard = np.isfinite(ref)
    err = np.abs(got[heard] - ref[heard])
    print("pair sums |error| p50, p99, max (dB):", np.percentile(err, [50, 99, 100]))
    assert err.max() < TOL_DB, np.percentile(err, [50, 99, 100])
    assert np.median(err) < 0.005
    got_p, ref_p = _levels_db(points.astype(np.float64)), _levels_db(ref_points)
    assert np.array_equal(np.isfinite(got_p), np.isfinite(ref_p))
    heard = np.isfinite(ref_p)
    pe = np.abs(got_p[heard] - ref_p[heard])
    assert pe.max() < TOL_DB, np.percentile(pe, [50, 99, 100])


def test_pairs_match_the_oracle_on_the_road_square(ctx, road):
    _check_pairs(ctx, road[0], np.random.default_rng(9))


def test_pairs_match_the_oracle_on_the_terrain_square(ctx, terrain):
    _check_pairs(ctx, terrain[0], np.random.default_rng(10))


def test_zwicker_matches_the_oracle(ctx):
    rng = np.random.default_rng(11)
    levels = rng.uniform(-10.0, 95.0, (20000, 28))
    levels[::7, :6] = -np.inf
    levels[::11] = rng.uniform(-80.0, 20.0, 28)
    sone = ctx.zwicker(levels.astype(np.float32))
    ref = oracle.zwicker_many(levels.astype(np.float32).astype(np.float64))
    big = ref > 1e-3
    rel = np.abs(sone[big] - ref[big]) / ref[big]
    assert rel.max() < 0.005, rel.max()
    assert np.all(np.abs(sone[~big] - ref[~big]) < 1e-4)


def test_level_histogram_counts_are_exact(ctx):
    rng = np.random.default_rng(12)
    levels = rng.uniform(-60.0, 200.0, 200000).astype(np.float32)
    levels[:100] = np.round(levels[:100] * 20) / 20  # half-bin boundaries
    levels[100] = np.nan
    levels[101] = -np.inf
    counts = ctx.level_histogram(levels)
    ref = oracle.level_histogram(levels.astype(np.float64), -30.0, 0.1, 1800)
    np.testing.assert_array_equal(counts, ref)


def _point_sources(stock, points_m, level_db=90.0, height_m=0.05):
    from quietmap_b200 import abi
    src = np.zeros(len(points_m), dtype=abi.SOURCE_DTYPE)
    for k, p in enumerate(points_m):
        x, y = stock.steps(p)
        src[k]["x"], src[k]["y"] = x, y
        src[k]["height_m"] = height_m
        src[k]["ground_factor"] = -1.0
        src[k]["energy"][:] = 10.0 ** (level_db / 10.0)
    return src


def test_over_capacity_paths_are_rerun_on_the_device(ctx):
    """140 buildings in a row: rays along it cross 280 walls, beyond the painter's per-path
    capacity; those paths are re-run with large capacities and still match the oracle."""
    stock = Stock(side_m=2600.0, offset_m=200.0)
    for i in range(140):
        stock.building(i + 1, 3.0 + (i % 7), [square(100.0 + 12.0 * i, 0.0, 5.0)])
    sources = _point_sources(stock, [(40.0, 0.0), (40.0, 1.5), (45.0, -2.0), (60.0, 30.0)])
    scene = stock.scene(sources=sources)
    origin = stock.steps((1900.0, -12.0))
    grid = scenes.Grid(origin=tuple(int(v) for v in origin), spacing=int(round(2.0 / stock.step_m)), nx=8, ny=12)
    dev = ctx.scene(scene)
    bands, dba, lden, hist, stats = dev.paint_grid(grid)
    assert stats["failed_paths"] > 0, stats
    ora = oracle.OracleScene(scene)
    e, l, _ = ora.paint_grid(grid)
    ref = _levels_db(e.sum(axis=1))
    np.testing.assert_allclose(dba, ref, atol=TOL_DB)
