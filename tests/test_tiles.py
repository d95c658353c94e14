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
