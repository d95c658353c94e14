"""Tile batches on the host: the uneven-tile generator and the bucket and default-table rules of
the C ABI (host functions; no device needed)."""

import numpy as np

from quietmap_b200 import abi, native, scenes


def test_uneven_tiles_follow_their_distributions():
    world = scenes.tiles_world()
    tiles = scenes.uneven_tiles(world, n_tiles=4096)
    assert len(tiles) == 4096
    nx = np.array([t["nx"] for t in tiles])
    src = np.array([t["source_end"] - t["source_begin"] for t in tiles])
    assert nx.min() >= 32 and nx.max() <= 512
    assert src.min() >= 10 and src.max() <= 50000
    # log-uniform: about half the tiles below the geometric middle of each range
    assert abs(np.mean(nx < np.sqrt(32 * 512)) - 0.5) < 0.05
    assert abs(np.mean(src < np.sqrt(10 * 50000)) - 0.5) < 0.05
    # cells numbered tile after tile, receivers inside the scene
    offsets = np.array([t["cell_offset"] for t in tiles])
    cells = np.array([t["nx"] * t["ny"] for t in tiles])
    assert np.array_equal(offsets[1:], np.cumsum(cells)[:-1])
    ext = world.extent_steps[0]
    for t in tiles[:200]:
        assert t["origin"][0] + (t["nx"] - 1) * t["spacing"] < ext
        assert t["source_end"] <= len(world.sources)


def test_tile_buckets_and_default_table():
    def tile(nx, ny):
        return dict(origin=(0, 0), spacing=1, nx=nx, ny=ny, source_begin=0, source_end=1, cell_offset=0)
    assert native.tile_bucket(tile(32, 40)) == 0
    assert native.tile_bucket(tile(63, 10)) == 0
    assert native.tile_bucket(tile(64, 10)) == 1
    assert native.tile_bucket(tile(10, 200)) == 2
    assert native.tile_bucket(tile(512, 300)) == 3
    t = native.tune_default()
    for b in range(abi.TILE_BUCKETS):
        c = t.bucket[b]
        assert (c.block_w, c.block_h, c.threads, c.chunk) == (16, 8, 128, 512)


def test_uneven_tile_specs_follow_their_distributions():
    specs = scenes.uneven_tile_specs(n_tiles=4096)
    nx = np.array([s["nx"] for s in specs])
    seg = np.array([s["segments"] for s in specs])
    bld = np.array([s["buildings"] for s in specs])
    assert nx.min() >= 32 and nx.max() <= 512 and seg.min() >= 10 and seg.max() <= 50000
    assert bld.min() == 0 and bld.max() <= 20000
    assert abs(np.mean(nx < np.sqrt(32 * 512)) - 0.5) < 0.05
    assert abs(np.mean(seg < np.sqrt(10 * 50000)) - 0.5) < 0.05
    assert abs(np.mean(bld + 1 < np.sqrt(20001)) - 0.5) < 0.05


def test_uneven_tile_world_gives_each_tile_its_own_region_roads_and_buildings():
    specs = scenes.uneven_tile_specs(n_tiles=4096)
    pick = [specs[k] for k in (3, 17, 40, 41)]
    scene, tiles = scenes.uneven_tile_world(pick, max_paths_per_tile=1 << 24)
    assert len(tiles) == 4
    assert sum(t["buildings"] for t in tiles) == len(scene.outlines)
    offsets = [t["cell_offset"] for t in tiles]
    assert offsets == list(np.cumsum([0] + [t["nx"] * t["ny"] for t in tiles[:-1]]))
    boxes = []
    for t, sp in zip(tiles, pick):
        src = scene.sources[t["source_begin"]:t["source_end"]]
        assert t["nx"] * t["ny"] * len(src) <= (1 << 24) + t["nx"] * t["ny"] * 200
        assert t["kept_segments"] <= sp["segments"] and t["buildings"] <= sp["buildings"]
        x0 = min(src["x"].min(), t["origin"][0])
        x1 = max(src["x"].max(), t["origin"][0] + (t["nx"] - 1) * t["spacing"])
        y0 = min(src["y"].min(), t["origin"][1])
        y1 = max(src["y"].max(), t["origin"][1] + (t["ny"] - 1) * t["spacing"])
        boxes.append((x0, x1, y0, y1))
    # The tiles' regions do not overlap: a tile's rays meet only its own buildings.
    for i in range(4):
        for j in range(i + 1, 4):
            a, b = boxes[i], boxes[j]
            assert a[1] < b[0] or b[1] < a[0] or a[3] < b[2] or b[3] < a[2]
    assert scene.vertices.max() < scene.extent_steps[0]
