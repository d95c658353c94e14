"""The reference's packed per-pixel loudness input (paint/src/sone.rs:32-51, 217-234) read by the
library (qm_pixel_read): a pixel packed here by the format's rule (per layer its steady energy,
line count and 43-float lines; then each layer's curves and the place's, 28 floats per period)
reads back line by line for every period as float32 values, profiles and missing duties or
passes included; curves without a shape are marked; malformed pixels are refused."""

import math

import numpy as np
import pytest

from quietmap_b200 import abi, native

LAYERS = 6
STATES = abi.WEATHER_STATES


def _pack(layers, curves):
    """layers: [(steady[3], [line dicts])]; curves: [n_layers + 1][3] shapes (28 dB) or None."""
    out = []
    for steady, lines in layers:
        out += list(steady) + [float(len(lines))]
        for line in lines:
            out += list(line["energy"])
            for period in range(3):
                out += list(line["means"][period])
            out += list(line["lambda"])
            out.append(-1.0 if line["profile"] is None else float(line["profile"]))
            for key in ("duty", "passing"):
                out += [math.nan] * 3 if line[key] is None else list(line[key])
    for per_period in curves:
        for shape in per_period:
            out += [math.nan] * 28 if shape is None else list(shape)
    return np.array(out, dtype=np.float32)


def _pixel(rng):
    layers = []
    for layer in range(LAYERS):
        lines = []
        for _ in range(int(rng.integers(0, 5)) if layer != 4 else 0):
            kind = rng.integers(0, 4)
            lines.append(dict(
                energy=list(10.0 ** rng.uniform(2.0, 7.0, 3)),
                means=[list(10.0 ** rng.uniform(2.0, 7.0, STATES)) for _ in range(3)],
                **{"lambda": list(10.0 ** rng.uniform(-3.0, 3.0, 3))},
                profile=None if kind == 0 else int(rng.integers(0, 12)),
                duty=list(rng.uniform(0.0, 0.3, 3)) if kind == 1 else None,
                passing=list(rng.uniform(0.0, 5.0, 3)) if kind == 2 else None))
        layers.append((list(10.0 ** rng.uniform(0.0, 6.0, 3)), lines))
    curves = [[None if rng.random() < 0.2 else list(rng.uniform(-60.0, 5.0, 28)) for _ in range(3)]
              for _ in range(LAYERS + 1)]
    return layers, curves


def test_a_packed_pixel_reads_back_for_every_period():
    rng = np.random.default_rng(21)
    for _ in range(20):
        layers, curves = _pixel(rng)
        packed = _pack(layers, curves)
        f32 = lambda v: float(np.float32(v))
        for period in range(3):
            lines, profiles, steady, shapes, has_shape = native.pixel_read(packed, LAYERS, period)
            expected = [(layer, line) for layer, (_, ls) in enumerate(layers) for line in ls]
            assert len(lines) == len(expected)
            for row, profile, (layer, line) in zip(lines, profiles, expected):
                assert row["layer"] == layer and row["energy"] == f32(line["energy"][period])
                assert np.array_equal(row["means"], np.float32(line["means"][period]).astype(np.float64))
                assert row["lambda"] == f32(line["lambda"][period])
                assert profile == (-1 if line["profile"] is None else line["profile"])
                for key in ("duty", "passing"):
                    if line[key] is None:
                        assert math.isnan(row[key])
                    else:
                        assert row[key] == f32(line[key][period])
            assert np.array_equal(steady, [f32(st[period]) for st, _ in layers])
            for c in range(LAYERS + 1):
                shape = curves[c][period]
                assert has_shape[c] == (shape is not None)
                if shape is not None:
                    assert np.array_equal(shapes[c], np.float32(shape).astype(np.float64))
            # The lines read go straight into a period's layers.
            native.distribution_layers(2.0, lines, steady)


def test_malformed_pixels_are_refused():
    rng = np.random.default_rng(2)
    layers, curves = _pixel(rng)
    packed = _pack(layers, curves)
    for cut, words in ((packed[:-1], "curve 6"), (np.concatenate([packed, [0.0]]), "left over")):
        with pytest.raises(native.QmError) as err:
            native.pixel_read(cut, LAYERS, 0)
        assert err.value.status == abi.QM_ERR_ARGUMENT and words in str(err.value)
    bad = packed.copy()
    bad[3] = 2.5
    with pytest.raises(native.QmError) as err:
        native.pixel_read(bad, LAYERS, 0)
    assert "no whole line count" in str(err.value)
    bad[3] = 1e6
    with pytest.raises(native.QmError) as err:
        native.pixel_read(bad, LAYERS, 0)
    assert "runs past" in str(err.value)
    total = sum(len(ls) for _, ls in layers)
    if total > 1:
        with pytest.raises(native.QmError) as err:
            native.pixel_read(packed, LAYERS, 0, cap=1)
        assert err.value.status == abi.QM_ERR_CAPACITY
    with pytest.raises(native.QmError):
        native.pixel_read(packed, LAYERS, 3)


def _oracle_layers(layers, f32=lambda v: float(np.float32(v))):
    from oracle import distribution as dist

    out = []
    for steady, lines in layers:
        made = []
        for line in lines:
            made.append((dist.Line([f32(v) for v in line["energy"]],
                                   [[f32(v) for v in period] for period in line["means"]],
                                   [f32(v) for v in line["lambda"]],
                                   duty=None if line["duty"] is None else [f32(v) for v in line["duty"]],
                                   passing=None if line["passing"] is None else [f32(v) for v in line["passing"]]),
                         line["profile"]))
        out.append(([f32(v) for v in steady], made))
    return out


@pytest.mark.parametrize("runs", [None, (4, 1, 3)])
def test_a_packed_pixels_distributions_match_the_oracle(runs):
    """A packed pixel's layers and place, every period, on the map's 2 dB grid, with its profiled
    roads over the period's hours apart or in the map's groups: equal to the oracle's composition
    of the same float32 values to the bit (sparse lines' Kurze values included: on these pixels the
    library's sampler and the oracle's agree exactly)."""
    from oracle import distribution as dist

    rng = np.random.default_rng(23)
    shares = rng.uniform(0.3, 9.0, (12, 24))
    for trial in range(6):
        layers, curves = _pixel(rng)
        packed = _pack(layers, curves)
        got_layers, got_silent, got_place, got_place_silent = native.pixel_distributions(
            packed, LAYERS, 2.0, shares, None if runs is None else list(runs))
        made = _oracle_layers(layers)
        profiled = any(profile is not None for _, lines in made for _, profile in lines)
        groups = None
        if profiled:
            groups = []
            for p in range(3):
                slots_of, hours = dist.hour_groups(shares.tolist(), p, None if runs is None else runs[p])
                parts = []
                for slots in slots_of:
                    per_layer = []
                    for _, lines in made:
                        if not any(profile is not None for _, profile in lines):
                            per_layer.append(None)
                        else:
                            per_layer.append([1.0 if profile is None else
                                              dist.group_factor(shares.tolist(), profile, p, slots)
                                              for _, profile in lines])
                    parts.append((len(slots), per_layer))
                groups.append((hours, parts))
        each, whole = dist.layered_distributions([([line for line, _ in lines], steady) for steady, lines in made],
                                                 2.0, groups)

        def close(got, silent, want):
            want_bins = np.array(want.bins).reshape(-1, 2)
            assert np.array_equal(got, want_bins) and silent == want.silent

        for p in range(3):
            close(got_place[p], got_place_silent[p], whole[p])
            for layer in range(LAYERS):
                close(got_layers[layer, p], got_silent[layer, p], each[layer][p])


def test_a_pixel_naming_an_unknown_profile_is_refused():
    rng = np.random.default_rng(3)
    layers, curves = _pixel(rng)
    if not any(line["profile"] is not None for _, lines in layers for line in lines):
        layers[0][1].append(dict(energy=[1.0] * 3, means=[[1.0] * STATES] * 3, profile=0, duty=None,
                                 passing=None, **{"lambda": [20.0] * 3}))
    with pytest.raises(native.QmError) as err:
        native.pixel_distributions(_pack(layers, curves), LAYERS, 2.0, np.ones((0, 24)), None)
    assert err.value.status == abi.QM_ERR_ARGUMENT and "profile" in str(err.value)


def test_a_packed_pixels_ndens_match_the_oracle():
    """Nden per layer and for the place: each layer's distributions on its own curves, the place's
    on the place's (curves from the packed shapes, the loudness at each whole decibel by the
    oracle's Zwicker), equal to the oracle's loudness of its composition to the bit; a layer
    without a shape reads 0."""
    from oracle import distribution as dist
    from oracle import oracle

    rng = np.random.default_rng(29)
    shares = rng.uniform(0.3, 9.0, (12, 24))
    layers, curves = _pixel(rng)
    curves[2] = [None, None, None]
    packed = _pack(layers, curves)
    tables = np.zeros((LAYERS + 1, 3, 191))
    oracle_curves = []
    for c in range(LAYERS + 1):
        per_period = []
        for p in range(3):
            curve = dist.Curve.__new__(dist.Curve)
            shape = curves[c][p]
            if shape is None:
                curve.table = [0.0] * 191
            else:
                shape32 = np.float32(shape).astype(np.float64)
                curve.table = list(oracle.zwicker_many([shape32 + (-30.0 + step) for step in range(191)]))
            tables[c, p] = curve.table
            per_period.append(curve)
        oracle_curves.append(per_period)
    got = native.pixel_ndens(packed, LAYERS, 2.0, tables, shares, [4, 1, 3])
    layer_bins, layer_silent, place_bins, place_silent = native.pixel_distributions(packed, LAYERS, 2.0, shares,
                                                                                    [4, 1, 3])
    for c in range(LAYERS + 1):
        bins = place_bins if c == LAYERS else layer_bins[c]
        distributions = []
        for p in range(3):
            d = dist.Distribution(2.0)
            d.bins = [list(row) for row in bins[p]]
            distributions.append(d)
        _, want = dist.loudness(distributions, oracle_curves[c])
        assert got[c] == want, c
    assert got[2] == 0.0 and got[LAYERS] > 0.0
