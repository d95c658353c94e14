"""Tile batches on the GPU: one persistent, graph-captured launch over uneven tiles against one
qm_paint_grid call per tile, and the autotuner."""

import numpy as np
import pytest

from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    ctx = native.Context(0)
    scene, full = scenes.road_square()
    dev = ctx.scene(scene)
    tiles = scenes.uneven_tiles(scene, n_tiles=10, seed=9, side=(8, 70), sources=(10, 3000), spacing_steps=256)
    return ctx, scene, dev, tiles


def _per_tile(dev, tiles, n_cells):
    dba = np.full(n_cells, -np.inf, np.float32)
    bands = np.full((n_cells, 8), -np.inf, np.float32)
    for t in tiles:
        g = scenes.Grid(origin=t["origin"], spacing=t["spacing"], nx=t["nx"], ny=t["ny"], height_m=t["height_m"],
                        source_begin=t["source_begin"], source_end=t["source_end"])
        b, d, _, _, _ = dev.paint_grid(g, histogram=False)
        o = t["cell_offset"]
        dba[o:o + g.cells] = d
        bands[o:o + g.cells] = b
    return bands, dba


def test_batch_matches_one_call_per_tile(setup):
    ctx, scene, dev, tiles = setup
    n_cells = tiles[-1]["cell_offset"] + tiles[-1]["nx"] * tiles[-1]["ny"] + 5  # 5 cells no tile covers
    plan = native.BatchPlan(dev, tiles, n_cells=n_cells)
    st = plan.run()
    bands, dba, lden = plan.read()
    assert st["paths"] == sum(t["nx"] * t["ny"] * (t["source_end"] - t["source_begin"]) for t in tiles)
    ref_bands, ref_dba = _per_tile(dev, tiles, n_cells)
    assert np.all(np.isneginf(dba[-5:]))
    np.testing.assert_allclose(dba[:-5], ref_dba[:-5], atol=0.01)
    np.testing.assert_allclose(bands[:-5], ref_bands[:-5], atol=0.01)


def test_graph_replays_are_bit_exact_and_shapes_agree(setup):
    ctx, scene, dev, tiles = setup
    graph = native.BatchPlan(dev, tiles)
    graph.run()
    a = graph.read()
    graph.run()
    b = graph.read()
    plain = native.BatchPlan(dev, tiles, graph=False)
    plain.run()
    c = plain.read()
    for x, y, z in zip(a, b, c):
        assert np.array_equal(x, y) and np.array_equal(x, z)
    # another launch shape (32x32 blocks of 256 threads, 128-source chunks) paints the same levels
    table = abi.TuneTable()
    for k in range(abi.TILE_BUCKETS):
        table.bucket[k] = abi.TileConfig(32, 32, 256, 128)
    other = native.BatchPlan(dev, tiles, table=table)
    other.run()
    np.testing.assert_allclose(other.read()[1], a[1], atol=0.01)


def test_autotune_picks_a_timed_candidate(setup):
    ctx, scene, dev, tiles = setup
    table, timings = native.autotune(dev, tiles[:4])
    buckets = {native.tile_bucket(t) for t in tiles[:4]}
    for b in range(abi.TILE_BUCKETS):
        c = table.bucket[b]
        if b in buckets:
            assert np.all(timings[b] > 0)
            k = int(np.argmin(timings[b]))
            assert c.chunk == [128, 256, 512, 1024, 2048][k % 5]
        else:
            assert np.all(timings[b] == -1)
            assert (c.block_w, c.chunk) == (16, 512)


def test_plans_mixing_thread_counts_keep_their_buffers(setup):
    """A table whose buckets use 128- and 256-thread CTAs gives a plan with two launches. Building
    it must not free the first launch's work list (it once did, when the launch list grew), so
    the plan paints the default plan's levels, frees cleanly, and later plans still capture."""
    ctx, scene, dev, tiles = setup
    buckets = {native.tile_bucket(t) for t in tiles}
    assert {0, 1} <= buckets
    table = abi.TuneTable()
    table.bucket[0] = abi.TileConfig(16, 8, 128, 512)
    for k in range(1, abi.TILE_BUCKETS):
        table.bucket[k] = abi.TileConfig(32, 32, 256, 128)
    ref = native.BatchPlan(dev, tiles)
    ref.run()
    ref_dba = ref.read()[1]
    ref.close()
    for _ in range(2):
        mixed = native.BatchPlan(dev, tiles, table=table)
        mixed.run()
        np.testing.assert_allclose(mixed.read()[1], ref_dba, atol=0.01)
        mixed.close()
    again = native.BatchPlan(dev, tiles)
    again.run()
    assert np.array_equal(again.read()[1], ref_dba)
    again.close()


def test_batch_of_tiles_each_with_its_own_roads_and_buildings():
    """Config 4's tiles: each its own roads and buildings in a region of its own; the batch paints
    them as one call per tile does, and a tile's levels come from its own scene only (a tile alone
    in a world of its own paints the same)."""
    ctx = native.Context(0)
    specs = scenes.uneven_tile_specs(n_tiles=64, seed=11, side=(16, 48), segments=(10, 60), buildings=(0, 400))
    world, tiles = scenes.uneven_tile_world(specs[:6], max_paths_per_tile=1 << 22)
    assert sum(t["buildings"] for t in tiles) > 0
    dev = ctx.scene(world)
    n_cells = tiles[-1]["cell_offset"] + tiles[-1]["nx"] * tiles[-1]["ny"]
    plan = native.BatchPlan(dev, tiles, n_cells=n_cells)
    plan.run()
    bands, dba, _ = plan.read()
    ref_bands, ref_dba = _per_tile(dev, tiles, n_cells)
    np.testing.assert_allclose(dba, ref_dba, atol=0.01)
    np.testing.assert_allclose(bands, ref_bands, atol=0.01)
    alone, alone_tiles = scenes.uneven_tile_world(specs[2:3], max_paths_per_tile=1 << 22)
    t = alone_tiles[0]
    g = scenes.Grid(origin=t["origin"], spacing=t["spacing"], nx=t["nx"], ny=t["ny"], source_begin=t["source_begin"],
                    source_end=t["source_end"])
    _, d_alone, _, _, _ = ctx.scene(alone).paint_grid(g, histogram=False)
    o = tiles[2]["cell_offset"]
    np.testing.assert_allclose(d_alone, dba[o:o + g.cells], atol=0.01)
    plan.close()
    ctx.close()
