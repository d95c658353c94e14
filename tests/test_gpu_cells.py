"""Map cells on the device (qm_quantize_cells) against the oracle: bytes identical, the reference's
known answers, and its errors (the lowest invalid pixel and layer, unassessed pixels unchecked)."""

import math

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, native

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = native.Context(0)
    yield c
    c.close()


def energy(level_db):
    return math.exp(level_db * (2.302585092994046 / 10.0))


def test_cells_are_byte_identical_to_the_oracle(ctx):
    rng = np.random.default_rng(21)
    n = 300_000
    layers = 10.0 ** rng.uniform(-4, 16, (n, abi.LAYERS))
    layers[rng.random((n, abi.LAYERS)) < 0.25] = 0.0
    sone = 2.0 ** rng.uniform(-7, 10, (n, abi.LAYERS + 1))
    sone[rng.random((n, abi.LAYERS + 1)) < 0.02] = 0.0
    sone[rng.random((n, abi.LAYERS + 1)) < 0.01] = np.nan
    sone[rng.random((n, abi.LAYERS + 1)) < 0.01] = np.inf
    assessed = (rng.random(n) > 0.1).astype(np.uint8)
    lc, nc = ctx.quantize_cells(layers, sone, assessed)
    rlc, rnc = oracle.quantize_cells(layers, sone, assessed)
    np.testing.assert_array_equal(lc, rlc)
    np.testing.assert_array_equal(nc, rnc)
    only, none = ctx.quantize_cells(layers)
    assert none is None
    np.testing.assert_array_equal(only, oracle.quantize_cells(layers)[0])


def test_known_answers_on_the_device(ctx):
    values = [0.0, energy(-0.01), 1.0, energy(60.26), energy(150.0), energy(60.0)]
    layers = np.array([values])
    lc, _ = ctx.quantize_cells(layers)
    assert list(lc[0, :abi.LAYERS]) == [abi.CELL_SILENCE, abi.CELL_SILENCE, 0, 121, 253, 120]
    two = np.zeros((1, abi.LAYERS))
    two[0, 0] = two[0, 5] = energy(60.0)
    assert ctx.quantize_cells(two)[0][0, abi.LAYERS] == 126
    sone = np.array([[1.0, 2.0, 0.5, 1.0 / 16.0, 0.06, np.nan, np.inf]])
    _, nc = ctx.quantize_cells(np.ones((1, abi.LAYERS)), sone)
    assert list(nc[0]) == [80, 100, 60, 0, abi.CELL_SILENCE, abi.CELL_SILENCE, 253]


def test_errors_name_the_lowest_bad_pixel_and_layer(ctx):
    layers = np.ones((64, abi.LAYERS))
    layers[40, 3] = -1.0
    layers[12, 2] = np.nan
    layers[12, 4] = np.inf
    with pytest.raises(native.QmError, match="pixel 12, layer 2: invalid Lden energy NaN"):
        ctx.quantize_cells(layers)
    assessed = np.ones(64, np.uint8)
    assessed[12] = 0
    with pytest.raises(native.QmError, match="pixel 40, layer 3"):
        ctx.quantize_cells(layers, assessed=assessed)
    over = np.full((2, abi.LAYERS), 1e308)
    with pytest.raises(native.QmError, match="pixel 0, total: invalid Lden energy inf"):
        ctx.quantize_cells(over)
    cells, _ = ctx.quantize_cells(over, assessed=np.zeros(2, np.uint8))
    assert np.all(cells == abi.CELL_NO_LEVEL)


def test_hm3_streams_match_the_oracle(ctx):
    rng = np.random.default_rng(22)
    y, x = np.mgrid[0:512, 0:512]
    smooth = np.clip(110 + 50 * np.sin(y / 41.0) * np.cos(x / 29.0) + rng.normal(0, 2, (512, 512)), 0, 253)
    tiles = np.stack([rng.integers(0, 256, (512, 512)), smooth, np.full((512, 512), 254), (x + 3 * y) % 256,
                      rng.integers(0, 2, (512, 512)) * 255]).astype(np.uint8)
    tiles[1, 200:260, 40:90] = 255
    layers = np.array([0, 3, 6, 5, 1], np.uint8)
    for metric in (0, 1):
        got = ctx.hm3_predict(tiles, layers, metric)
        for k in range(len(tiles)):
            np.testing.assert_array_equal(got[k], oracle.hm3_predict(tiles[k], layers[k], metric))
    with pytest.raises(native.QmError, match="unknown layer 7"):
        ctx.hm3_predict(tiles[:1], np.array([7], np.uint8), 0)
    with pytest.raises(native.QmError, match="metric"):
        ctx.hm3_predict(tiles[:1], layers[:1], 2)
