"""`terrain` tiles (qmterr2): the library's decoder against tiles the oracle writes, pinned to the
reference's own decode test (tiles/src/terrain.rs:438-473). Host only."""

import math

import numpy as np
import pytest

from oracle import terrain as ot
from quietmap_b200 import native


def _xorshift(seed):
    mask = (1 << 64) - 1
    while True:
        seed ^= (seed << 13) & mask
        seed ^= seed >> 7
        seed ^= (seed << 17) & mask
        yield seed


def _reference_nodes(rows, columns):
    """The reference test's nodes: random heights (steep jumps, the missing code and the u16
    ends wrap the prediction), percents and canopies, from its own generator and seed."""
    draw = _xorshift(0x9E37_79B9_7F4A_7C15)
    heights = np.zeros(rows * columns, np.uint16)
    imp, forest, canopy = (np.zeros(rows * columns, np.uint8) for _ in range(3))
    for at in range(rows * columns):
        kind = next(draw) % 7
        if kind == 0:
            heights[at] = ot.HEIGHT_MISSING
        elif kind == 1:
            heights[at] = 0
        elif kind == 2:
            heights[at] = next(draw) % 65_536
        else:
            heights[at] = (2_500 + (at % 65_536 % 53) * 3 + next(draw) % 5) & 0xFFFF
        imp[at] = next(draw) % 101
        forest[at] = next(draw) % 102
        canopy[at] = next(draw) % 61
    shape = (rows, columns)
    return heights.reshape(shape), imp.reshape(shape), forest.reshape(shape), canopy.reshape(shape)


def test_a_tile_decodes_to_the_nodes_it_was_encoded_from():
    heights, imp, forest, canopy = _reference_nodes(37, 53)
    data = ot.encode(181_042, 50_625, heights, imp, forest, canopy)
    window, h, i, f, c = native.terrain_decode(data)
    assert window == dict(north_node=181_042, west_node=50_625, rows=37, columns=53)
    np.testing.assert_array_equal(h, heights)
    np.testing.assert_array_equal(i, imp)
    np.testing.assert_array_equal(f, forest)
    np.testing.assert_array_equal(c, canopy)


def test_broken_tiles_are_refused():
    heights, imp, forest, canopy = _reference_nodes(4, 5)
    data = ot.encode(180_001, 50_000, heights, imp, forest, canopy)
    native.terrain_decode(data)
    with pytest.raises(native.QmError, match="does not decode"):
        native.terrain_decode(data[:-1])
    with pytest.raises(native.QmError, match="bad magic"):
        native.terrain_decode(b"qmterr1\n" + data[8:])
    for rows, columns in ((0, 5), (4, 1025)):
        bad = bytearray(data)
        bad[16:20] = rows.to_bytes(4, "little")
        bad[20:24] = columns.to_bytes(4, "little")
        with pytest.raises(native.QmError, match="a window no tile has"):
            native.terrain_decode(bytes(bad))
    short = data[:24] + ot.compress(ot.planes(heights, imp, forest, canopy)[:-5])
    with pytest.raises(native.QmError, match="does not match the window"):
        native.terrain_decode(short)


def test_a_fine_tile_decodes_to_the_details_it_was_encoded_from():
    """tiles/src/terrain_fine.rs:286-330: blocks of every shape (2.3 blocks by 1.5), negative and
    positive details and the i16 ends; a cut tile and a bad frame are errors."""
    rows, columns = 2 * 128 + 40, 128 + 65
    at = np.arange(rows * columns)
    k = at % 97
    details = np.where(k == 0, -32768, np.where(k == 1, 32767, (k - 48) * 3 + (at // 300) % 7)).astype(np.int16)
    details = details.reshape(rows, columns)
    data = ot.encode_fine(1_076_760, 307_800, details)
    window, got = native.terrain_fine_decode(data)
    assert window == dict(north_node=1_076_760, west_node=307_800, rows=rows, columns=columns)
    np.testing.assert_array_equal(got, details)
    with pytest.raises(native.QmError, match="terrain-fine"):
        native.terrain_fine_decode(data[:24 + 8])
    broken = bytearray(data)
    broken[-1] ^= 0xFF
    with pytest.raises(native.QmError, match="a block does not decode"):
        native.terrain_fine_decode(bytes(broken))
    small = np.array([[0, 5, 10], [15, 20, 25], [30, 35, -40]], np.int16)
    assert np.array_equal(native.terrain_fine_decode(ot.encode_fine(6, 0, small))[1], small)
    with pytest.raises(native.QmError, match="a window no tile has"):
        native.terrain_fine_decode(ot.encode_fine(6, 0, small[:1]))


def _mercator_to_degrees(x, y):
    """tiles/src/geo.rs:43-47."""
    n = 4096.0
    lat = math.degrees(math.atan(math.sinh(math.pi * (1.0 - 2.0 * y / n))))
    return lat, x / n * 360.0 - 180.0


def test_prague_tile_window_brackets_the_tile():
    """tiles/src/terrain.rs:392-405."""
    x, y = native.mercator_from_degrees(50.07553, 14.43781)
    tile = (int(math.floor(x)), int(math.floor(y)))
    window = native.terrain_window_of_tile(*tile)
    assert 204 <= window["rows"] <= 207 and 318 <= window["columns"] <= 320, window
    north, west = _mercator_to_degrees(tile[0], tile[1])  # the tile's north-west corner
    assert window["north_node"] >= north * 3600.0 and window["west_node"] <= west * 3600.0


def test_columns_wrap_across_the_antimeridian():
    """tiles/src/terrain.rs:407-422."""
    west, east = native.terrain_window_of_tile(0, 2241), native.terrain_window_of_tile(4095, 2241)
    world, just_west = 4096.0, -0.001
    column = native.terrain_column_of(east, just_west)
    assert 0.0 <= column < east["columns"], column
    assert abs(native.terrain_column_of(east, world + just_west) - column) < 1e-6
    assert 0.0 <= native.terrain_column_of(west, 0.001) < west["columns"]
    assert abs(native.terrain_column_of(west, 0.001) - native.terrain_column_of(west, world + 0.001)) < 1e-6


def test_neighbours_share_their_seam_nodes():
    """tiles/src/terrain.rs:424-435."""
    here, east, south = (native.terrain_window_of_tile(2212, 1387), native.terrain_window_of_tile(2213, 1387),
                         native.terrain_window_of_tile(2212, 1388))
    assert here["west_node"] + here["columns"] > east["west_node"]
    assert here["north_node"] - here["rows"] < south["north_node"]


def test_samples_interpolate_heights_and_refuse_missing_nodes():
    """tiles/src/terrain.rs:475-517, through a tile the oracle writes and the library decodes."""
    code = lambda metres: int((metres + 500.0) * 5.0)
    heights = np.array([[code(100.0), code(110.0)], [code(120.0), code(130.0)]], np.uint16)
    imp = np.array([[0, 100], [0, 100]], np.uint8)
    forest = np.array([[0, 0], [80, 80]], np.uint8)
    canopy = forest // 4
    window, h, i, f, c = native.terrain_decode(ot.encode(180_001, 50_000, heights, imp, forest, canopy))
    at = lambda lat_nodes, lon_nodes: native.mercator_from_degrees(lat_nodes / 3600.0, lon_nodes / 3600.0)
    points = [at(180_000.5, 50_000.5), at(180_001.0, 50_000.0), at(180_000.5, 50_001.5), at(180_001.5, 50_000.5)]
    middle, north_west, east, north = native.terrain_sample(window, h, i, f, c, points)
    assert abs(middle["height_m"] - 115.0) < 1e-4 and abs(middle["ground_factor"] - 0.5) < 1e-5, middle
    assert abs(north_west["height_m"] - 100.0) < 1e-4 and north_west["forest_cover"] == 0.0
    assert east is None and north is None
    h[1, 1] = ot.HEIGHT_MISSING
    assert native.terrain_sample(window, h, i, f, c, points[:1]) == [None]
