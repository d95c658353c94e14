"""Map cells (the bytes `PaintedCells::from_painted` writes, paint/src/levels.rs): the oracle pinned
to the reference's known answers (levels.rs:115-137) and to the loudness cell's definition
(levels.rs:22-33: twice the loudness level in phon, 40 + 10 log2 sone)."""

import math

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi

ROAD, RAILWAY, AIRCRAFT = 0, 1, 5  # tiles/src/sources.rs:59-66


def energy(level_db):
    """physics/src/bands.rs:34-36: exp(L ln10 / 10)."""
    return math.exp(level_db * (2.302585092994046 / 10.0))


def test_lden_cells_match_the_reference_known_answers():
    assert oracle.lden_cell(0.0) == abi.CELL_SILENCE
    assert oracle.lden_cell(energy(-0.01)) == abi.CELL_SILENCE
    assert oracle.lden_cell(1.0) == 0
    assert oracle.lden_cell(energy(60.26)) == 121
    assert oracle.lden_cell(energy(150.0)) == 253
    for bad in (-1.0, math.inf, math.nan):
        with pytest.raises(ValueError):
            oracle.lden_cell(bad)


def test_layers_are_summed_before_the_logarithm():
    layers = np.zeros((13, abi.LAYERS))
    layers[12, ROAD] = energy(60.0)
    layers[12, AIRCRAFT] = energy(60.0)
    cells, _ = oracle.quantize_cells(layers)
    assert cells[12, abi.LAYERS] == 126
    assert cells[12, RAILWAY] == abi.CELL_SILENCE
    assert cells[12, ROAD] == 120
    layers[12, 2] = math.nan
    with pytest.raises(ValueError, match="pixel 12, layer 2"):
        oracle.quantize_cells(layers)


def test_a_total_that_overflows_is_an_error_and_unassessed_pixels_are_not_checked():
    layers = np.full((3, abi.LAYERS), 1e308)
    with pytest.raises(ValueError, match="pixel 0, total"):
        oracle.quantize_cells(layers)
    cells, _ = oracle.quantize_cells(layers, assessed=np.zeros(3, np.uint8))
    assert np.all(cells == abi.CELL_NO_LEVEL)


def test_loudness_cells_follow_the_definition():
    # 1 sone = 40 phon -> 80; a doubling is 20 steps; 1/16 sone = 0 phon -> 0; below: silence.
    assert [oracle.nden_cell(s) for s in (1.0, 2.0, 0.5, 1.0 / 16.0)] == [80, 100, 60, 0]
    assert oracle.nden_cell(0.06) == abi.CELL_SILENCE
    assert oracle.nden_cell(0.0) == abi.CELL_SILENCE
    assert oracle.nden_cell(math.nan) == abi.CELL_SILENCE
    assert oracle.nden_cell(-1.0) == abi.CELL_SILENCE
    assert oracle.nden_cell(math.inf) == 253
    assert oracle.nden_cell(2.0 ** 8.6) == 252


def test_pixels_quantize_per_layer_and_in_total():
    rng = np.random.default_rng(3)
    n = 2000
    layers = 10.0 ** rng.uniform(-3, 15, (n, abi.LAYERS))
    layers[rng.random((n, abi.LAYERS)) < 0.2] = 0.0
    sone = 2.0 ** rng.uniform(-6, 9, (n, abi.LAYERS + 1))
    assessed = (rng.random(n) > 0.1).astype(np.uint8)
    lc, nc = oracle.quantize_cells(layers, sone, assessed)
    for p in range(0, n, 97):
        if not assessed[p]:
            assert np.all(lc[p] == abi.CELL_NO_LEVEL) and np.all(nc[p] == abi.CELL_NO_LEVEL)
            continue
        assert [oracle.lden_cell(e) for e in layers[p]] == list(lc[p, :abi.LAYERS])
        assert oracle.lden_cell(sum(layers[p])) == lc[p, abi.LAYERS]
        assert [oracle.nden_cell(s) for s in sone[p]] == list(nc[p])


# HM3 / HMD streams before Brotli (paint/src/hm3.rs:68-109).

def _neighbourhood(left, above, corner, cell=100):
    """A tile whose pixel (1, 1) has the given left, above and upper-left neighbours."""
    t = np.zeros((512, 512), np.uint8)
    t[0, 0], t[0, 1], t[1, 0], t[1, 1] = corner, above, left, cell
    return t


@pytest.mark.parametrize("left,above,corner,predicted", [
    (10, 10, 10, 10),   # all equal: left
    (5, 15, 10, 10),    # the corner is nearest the estimate
    (20, 10, 0, 20),    # left nearest
    (10, 20, 0, 20),    # above nearest
    (10, 10, 0, 10),    # left and above tie: left
    (0, 30, 10, 30),    # above and corner tie: above
])
def test_paeth_prediction_follows_the_png_tie_order(left, above, corner, predicted):
    stream = oracle.hm3_predict(_neighbourhood(left, above, corner), 2, 1)
    assert stream[6 + 512 + 1] == (100 - predicted) % 256


def test_streams_start_with_their_header_and_edges_use_zeros():
    rng = np.random.default_rng(4)
    tile = rng.integers(0, 256, (512, 512), dtype=np.uint8)
    nden = oracle.hm3_predict(tile, 6, 0)
    lden = oracle.hm3_predict(tile, 0, 1)
    assert bytes(nden[:6]) == b"HM3 \x07\x06" and bytes(lden[:6]) == b"HMD \x01\x00"
    assert np.array_equal(nden[6:], lden[6:])
    r = nden[6:].reshape(512, 512)
    assert r[0, 0] == tile[0, 0]
    np.testing.assert_array_equal(r[0, 1:], tile[0, 1:] - tile[0, :-1])          # first row: left
    col = tile[:, 0].astype(np.int16)
    np.testing.assert_array_equal(r[1:, 0], (col[1:] - col[:-1]).astype(np.uint8))  # first column: above
    with pytest.raises(ValueError):
        oracle.hm3_predict(tile, 7, 0)


def test_residuals_invert_to_the_cells():
    rng = np.random.default_rng(5)
    smooth = np.clip(120 + 40 * np.sin(np.arange(512)[:, None] / 37.0) * np.cos(np.arange(512) / 23.0), 0, 253)
    tiles = [rng.integers(0, 256, (512, 512), dtype=np.uint8), smooth.astype(np.uint8),
             np.full((512, 512), abi.CELL_SILENCE, np.uint8)]
    tiles[1][100:140, 300:380] = abi.CELL_NO_LEVEL
    for t in tiles:
        np.testing.assert_array_equal(oracle.hm3_unpredict(oracle.hm3_predict(t, 1, 0)[6:]), t)


def test_the_library_restores_cells_from_a_stream():
    from quietmap_b200 import native
    rng = np.random.default_rng(6)
    y, x = np.mgrid[0:512, 0:512]
    tiles = [rng.integers(0, 256, (512, 512), dtype=np.uint8),
             np.clip(100 + 60 * np.sin(y / 33.0) * np.cos(x / 47.0), 0, 253).astype(np.uint8)]
    for metric in (0, 1):
        for t in tiles:
            stream = oracle.hm3_predict(t, 4, metric)
            np.testing.assert_array_equal(native.hm3_unpredict(stream, 4, metric), t)
    stream = oracle.hm3_predict(tiles[0], 4, 0)
    for layer, metric, data in ((3, 0, stream), (4, 1, stream), (4, 0, stream[:-1])):
        with pytest.raises(native.QmError, match="not this layer's HM3 tile"):
            native.hm3_unpredict(data, layer, metric)
    with pytest.raises(native.QmError, match="unknown HM3 layer"):
        native.hm3_unpredict(stream, 7, 0)


def test_every_byte_and_row_boundary_round_trips():
    """paint/src/hm3_tests.rs:22-39 without its Brotli stage: the stream's residuals come back to
    the cells; another layer or a cut stream is refused."""
    from quietmap_b200 import native
    at = np.arange(512 * 512)
    cells = ((at // 512 * 19 + at % 512 * 31) % 256).astype(np.uint8).reshape(512, 512)
    stream = oracle.hm3_predict(cells, 6, 0)
    np.testing.assert_array_equal(native.hm3_unpredict(stream, 6, 0), cells)
    np.testing.assert_array_equal(oracle.hm3_unpredict(stream[6:]), cells)
    with pytest.raises(native.QmError):
        native.hm3_unpredict(stream, 0, 0)
    with pytest.raises(native.QmError):
        native.hm3_unpredict(stream[:len(stream) // 2], 6, 0)
    with pytest.raises(native.QmError):
        native.hm3_unpredict(np.concatenate([stream, [0]]).astype(np.uint8), 6, 0)
