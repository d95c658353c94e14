"""The global weather table (qmwthr2): a place's favourable probabilities and air absorption,
pinned to the reference's own test (physics/src/weather.rs:236-276). Host only."""

import numpy as np
import pytest

from quietmap_b200 import abi, native
from quietmap_b200.physics import alpha_bands

ROWS, COLUMNS = 361, 720
NODE = abi.PERIODS * abi.SECTORS + 2 * abi.BANDS


def encode(percent, alpha_db_per_km):
    """The table's bytes (weather.rs:84-98): magic, then per node its percentages and its
    absorptions in 0.01 dB/km, rounded half away from zero (non-negative here)."""
    codes = np.floor(np.asarray(alpha_db_per_km) * 100.0 + 0.5).astype("<u2")
    nodes = np.concatenate([percent.reshape(-1, abi.PERIODS * abi.SECTORS).astype(np.uint8),
                            codes.reshape(-1, abi.BANDS).view(np.uint8)], axis=1)
    return b"qmwthr2\n" + nodes.tobytes()


def default_table():
    percent = np.zeros((ROWS * COLUMNS, abi.PERIODS, abi.SECTORS), np.uint8)
    alpha = np.tile(alpha_bands(15.0, 70.0), (ROWS * COLUMNS, 1))
    return percent, alpha


def at(lat, lon):
    return int((90.0 - lat) * 2.0) * COLUMNS + int(lon * 2.0) % COLUMNS


def test_the_table_interpolates_between_nodes_and_across_the_antimeridian(tmp_path):
    percent, alpha = default_table()
    percent[at(50.0, 0.0), 1, 3] = 40
    percent[at(50.0, 359.5), 1, 3] = 80
    alpha[at(50.0, 0.0), 7] = 100.0
    alpha[at(50.0, 359.5), 7] = 120.0
    table = encode(percent, alpha)
    assert len(table) == 8 + ROWS * COLUMNS * NODE
    p = lambda lat, lon: native.weather_place(table, lat, lon)[0][1, 3]
    assert abs(p(50.0, -0.25) - 0.6) < 1e-12
    assert abs(p(50.0, 359.75) - 0.6) < 1e-12
    assert abs(p(50.25, 0.0) - 0.2) < 1e-12
    assert abs(native.weather_place(table, 50.0, -0.25)[1][7] - 110.0) < 1e-9
    default = native.weather_place(table, 10.0, 10.0)[1]
    np.testing.assert_allclose(default, alpha_bands(15.0, 70.0), atol=0.005)
    with pytest.raises(native.QmError, match="bad magic or length"):
        native.weather_place(table[:100], 50.0, 0.0)
    # A click reads its four nodes from the file and gets the table's answer.
    path = tmp_path / "weather"
    path.write_bytes(table)
    for lat, lon in [(50.0, -0.25), (50.2, 359.9), (50.25, 0.0), (90.0, 10.0), (-90.0, 0.0)]:
        fav_file, alpha_file = native.weather_read_place(path, lat, lon)
        fav_mem, alpha_mem = native.weather_place(table, lat, lon)
        assert np.array_equal(fav_file, fav_mem) and np.array_equal(alpha_file, alpha_mem)
    path.write_bytes(table[:-1])
    with pytest.raises(native.QmError, match="bad magic or length"):
        native.weather_read_place(path, 50.0, 0.0)


def test_percentages_above_100_are_refused():
    percent, alpha = default_table()
    percent[12345, 2, 15] = 101
    table = encode(percent, alpha)
    with pytest.raises(native.QmError, match="a percentage above 100"):
        native.weather_place(table, 0.0, 0.0)


def test_sectors_interpolate_and_wrap_through_north():
    """physics/src/weather.rs:219-233, on the float row a scene stores (hence 1e-7)."""
    from oracle import oracle
    import math
    row = np.zeros(16, np.float32)
    row[0], row[15], row[4] = 0.8, 0.4, 0.6
    north = math.pi / 2
    assert abs(oracle.favourable_at(row, north) - 0.8) < 1e-7
    assert abs(oracle.favourable_at(row, 0.0) - 0.6) < 1e-7, "east is sector 4"
    assert abs(oracle.favourable_at(row, north + math.radians(11.25)) - 0.6) < 1e-7
