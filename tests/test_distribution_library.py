"""The library's level distributions (qm_distribution.cuh: one source for the host and the
device), run on the host through the C ABI: adding lines to distributions and reading exceeded
levels equal the oracle's restatement (pinned to the reference's distribution tests) to the bit
on 0.1, 0.5 and 2 dB grids; the reference's own properties hold through the library (passes
fill the time and keep the mean; many quiet lines keep their energy); line and pass values
match the oracle's; and the entry points reject what the reference cannot take."""

import math

import numpy as np
import pytest

from oracle import distribution as dist
from oracle import oracle
from quietmap_b200 import abi, native


def _bins(d):
    return np.array(d.bins, dtype=np.float64).reshape(-1, 2)


def _pairs(line):
    return np.array(line.pairs, dtype=np.float64).reshape(-1, 2)


def _lines(rng):
    """Lines of every kind the reference adds: Kurze lines sparse to dense, events over a duty,
    passes, steady sounds, values at zero, equal values, and random sets."""
    out = [(dist.line_values(lam), 10.0 ** rng.uniform(0.0, 7.0)) for lam in (1e-5, 1e-3, 0.05, 0.5, 3.0, 30.0)]
    out += [(dist.line_values(0.0, duty=d), 10.0 ** rng.uniform(0.0, 7.0)) for d in (0.001, 0.02, 0.5, 1.0)]
    out += [(dist.pass_values(m), 10.0 ** rng.uniform(0.0, 7.0)) for m in (1e-6, 0.01, 0.7, 5.0, 60.0)]
    out += [(dist.LineValues([(4e4, 1.0)]), 1.0), (dist.LineValues([(0.0, 0.3), (0.0, 0.7)]), 1.0),
            (dist.LineValues([(2.0, 0.25), (2.0, 0.25), (0.5, 0.5)]), 3.0)]
    for _ in range(10):
        n = int(rng.integers(1, 40))
        values = 10.0 ** rng.uniform(-3.0, 3.0, n) * (rng.random(n) > 0.1)
        shares = rng.dirichlet(np.ones(n))
        out.append((dist.LineValues(list(zip(values, shares))), 10.0 ** rng.uniform(-2.0, 9.0)))
    return out


@pytest.mark.parametrize("bin_db", [0.1, 0.5, 2.0])
def test_adding_lines_matches_the_oracle_to_the_bit(bin_db):
    rng = np.random.default_rng(int(bin_db * 10))
    ours = dist.Distribution(bin_db)
    ours.silent = 1.0
    bins, silent = _bins(ours), 1.0
    for line, scale in _lines(rng):
        want = ours.with_line(line, scale)
        got_bins, got_silent = native.distribution_with_line(bin_db, bins, silent, _pairs(line), scale)
        assert np.array_equal(got_bins, _bins(want)) and got_silent == want.silent
        for exceeded in (0.0, 0.01, 0.1, 0.5, 0.9, 0.999, 1.0):
            assert native.distribution_exceeded_db(bin_db, got_bins, exceeded) == want.exceeded_db(exceeded)
        # Values handed over in any order add the same: the library sorts them as the reference
        # does, equal values keeping their order.
        shuffled = _pairs(line)[rng.permutation(len(line.pairs))]
        again, again_silent = native.distribution_with_line(bin_db, bins, silent, shuffled, scale)
        assert np.allclose(again, got_bins, rtol=1e-12, atol=0.0) and abs(again_silent - got_silent) <= 1e-12
        ours, bins, silent = want, got_bins, got_silent
    assert np.count_nonzero(bins[:, 0]) > 10


def test_passes_in_progress_fill_the_time_and_keep_the_mean():
    """distribution.rs:308-338 through the library, and the values equal the oracle's."""
    for mean in (2.2250738585072014e-308, 1e-18, 1e-4, 0.03, 0.7, 5.0, 60.0, 700.0):
        values = native.distribution_pass_values(mean)
        assert np.all(np.isfinite(values)) and np.all(values[:, 1] >= 0.0), mean
        assert abs(values[:, 1].sum() - 1.0) < 1e-9 and abs((values[:, 0] * values[:, 1]).sum() - 1.0) < 1e-9, mean
        order = np.argsort(values[:, 0], kind="stable")
        assert np.array_equal(values[order], _pairs(dist.pass_values(mean))), mean
    sparse = native.distribution_pass_values(0.01)
    assert abs(sparse[0, 1] - 0.99005) < 1e-5 and sparse[1, 0] == 100.0


def test_many_quiet_lines_keep_their_energy():
    """distribution.rs:340-361 through the library: 500 lines at lambda 0.5 added one by one."""
    values = native.distribution_line_values(0.5)
    mean = float((values[:, 0] * values[:, 1]).sum())
    bins = np.zeros((native.distribution_bins(0.5), 2))
    silent = 1.0
    for _ in range(500):
        bins, silent = native.distribution_with_line(0.5, bins, silent, values)
    energy = float(bins[:, 1].sum())
    assert abs(energy / (500.0 * mean) - 1.0) < 1e-9, energy


def test_line_values_match_the_oracle():
    """Kurze lines by the library's sampler equal the oracle's within the sampler's 1e-12; events
    over a duty exactly; the node shares exactly."""
    for lam in (0.0, 1e-6, 1e-4, 2e-3, 0.5, 9.99, 10.0, 400.0, math.inf):
        got = native.distribution_line_values(lam)
        want = _pairs(dist.line_values(lam))
        nodes = np.array(dist.node_probabilities())
        assert len(got) == abi.DISTRIBUTION_LINE_NODES == len(nodes)
        assert np.array_equal(got[:, 1], nodes[:, 1])
        relative = np.array(oracle.relative_intensity(lam, list(nodes[:, 0])))
        assert np.allclose(got[:, 0], relative, rtol=1e-12, atol=0.0), lam
        assert np.allclose(np.sort(got[:, 0]), want[:, 0], rtol=1e-12, atol=0.0), lam
    for duty in (1e-3, 0.25, 1.0):
        assert np.array_equal(native.distribution_line_values(0.0, duty=duty), [[0.0, 1.0 - duty], [1.0 / duty, duty]])


def test_errors():
    bins = np.zeros((360, 2))
    for bin_db in (0.0, -1.0, math.nan, math.inf, 0.05, 400.0):
        with pytest.raises(native.QmError) as err:
            native.distribution_bins(bin_db)
        assert err.value.status == abi.QM_ERR_ARGUMENT, bin_db
    assert native.distribution_bins(0.1) == 1800 and native.distribution_bins(2.0) == 90
    for values in ([[-1.0, 1.0]], [[1.0, -0.5]], [[math.nan, 1.0]]):
        with pytest.raises(native.QmError) as err:
            native.distribution_with_line(0.5, bins, 1.0, values)
        assert err.value.status == abi.QM_ERR_ARGUMENT and "value 0" in str(err.value)
    with pytest.raises(native.QmError) as err:
        native.distribution_with_line(0.5, bins, 1.0, [[1.0, 1.0]], scale=0.0)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    with pytest.raises(native.QmError) as err:
        native.distribution_pass_values(800.0)
    assert err.value.status == abi.QM_ERR_ARGUMENT and "700" in str(err.value)
    with pytest.raises(native.QmError) as err:
        native.distribution_pass_values(60.0, cap=3)
    assert err.value.status == abi.QM_ERR_CAPACITY
    with pytest.raises(native.QmError) as err:
        native.distribution_line_values(0.5, duty=1.5)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    # A line of no values holds no time, so no moment survives the sum (as in the reference).
    start = np.zeros((360, 2))
    start[100] = (0.5, 0.5 * dist.energy(-30.0 + 100 * 0.5))
    out, silent = native.distribution_with_line(0.5, start, 0.5, np.zeros((0, 2)))
    assert np.array_equal(out, np.zeros((360, 2))) and silent == 0.0


def _period_rows(layers, period):
    """The library's rows for one period of the oracle's layers."""
    rows = []
    for index, (lines, _) in enumerate(layers):
        for line in lines:
            row = np.zeros((), dtype=abi.PERIOD_LINE_DTYPE)
            row["layer"] = index
            row["energy"] = line.energy[period]
            row["means"] = line.means[period]
            row["lambda"] = line.lam[period]
            row["duty"] = math.nan if line.duty is None else line.duty[period]
            row["passing"] = math.nan if line.passing is None else line.passing[period]
            rows.append(row)
    return np.array(rows, dtype=abi.PERIOD_LINE_DTYPE)


def _place(seed, sparse):
    """Layers of a random place: steady energy, roads whose means differ by weather state (dense,
    and with `sparse` also sparse Kurze lines), bells over a duty, flights in classes."""
    rng = np.random.default_rng(seed)
    states = dist.WEATHER_STATES
    e = dist.energy

    def road(level, lam):
        base = e(level)
        means = [[base * (1.0 + 0.3 * rng.random()) for _ in range(states)] for _ in range(3)]
        return dist.Line([base] * 3, means, lam)

    lams = [[20.0, 12.0, 10.0], [1e3, 50.0, 10.5]] + ([[0.03, 0.01, 0.002], [2.0, 1.0, 0.4], [8.0, 3.0, 0.9]]
                                                       if sparse else [])
    roads = ([road(rng.uniform(30.0, 65.0), lam) for lam in lams], [e(rng.uniform(20.0, 40.0))] * 3)
    bells = dist.Line([e(50.0)] * 3, [[e(50.0)] * states] * 3, [math.inf] * 3, duty=[0.05, 0.0, 0.01])
    events = ([bells], [0.0] * 3)
    classes = []
    for passing, level in ((0.02, 45.0), (0.4, 40.0), (80.0, 35.0), (1e-320, 50.0)):
        energy = [e(level), e(level - 3.0), 0.0]
        classes.append(dist.Line(energy, [[x] * states for x in energy], [math.inf] * 3,
                                 passing=[passing, passing * 0.5, 0.0]))
    planes = (classes, [0.0] * 3)
    quiet = ([], [e(25.0)] * 3)
    return [roads, events, planes, quiet]


@pytest.mark.parametrize("bin_db", [0.5, 2.0])
def test_layers_match_the_oracle_to_the_bit(bin_db):
    """A place of dense roads, bells, flights and a steady layer: every layer's distribution and
    the place's, each period, equal the oracle's to the bit."""
    layers = _place(3, sparse=False)
    each, whole = dist.layered_distributions(layers, bin_db)
    for p in range(3):
        got_each, got_silent, got_whole, got_whole_silent = native.distribution_layers(
            bin_db, _period_rows(layers, p), [steady[p] for _, steady in layers])
        for k in range(len(layers)):
            assert np.array_equal(got_each[k], _bins(each[k][p])) and got_silent[k] == each[k][p].silent, (p, k)
        assert np.array_equal(got_whole, _bins(whole[p])) and got_whole_silent == whole[p].silent, p


def test_layers_with_sparse_lines_match_the_oracle():
    """With sparse Kurze lines, whose values come from the library's sampler (within 1e-12 of the
    oracle's), every layer's and the place's mean intensity and exceeded levels stay within the
    sampler's agreement."""
    layers = _place(5, sparse=True)
    each, whole = dist.layered_distributions(layers, 0.5)
    for p in range(3):
        got_each, got_silent, got_whole, got_whole_silent = native.distribution_layers(
            0.5, _period_rows(layers, p), [steady[p] for _, steady in layers])
        pairs = [(got_each[k], got_silent[k], each[k][p]) for k in range(len(layers))]
        pairs.append((got_whole, got_whole_silent, whole[p]))
        for got, silent, want in pairs:
            mean = float(got[:, 1].sum())
            want_mean = sum(i * s for i, s in want.intensities())
            assert abs(mean - want_mean) <= 1e-9 * want_mean and abs(silent - want.silent) <= 1e-12
            for exceeded in (0.05, 0.1, 0.5, 0.9):
                level, want_level = native.distribution_exceeded_db(0.5, got, exceeded), want.exceeded_db(exceeded)
                assert level == want_level or abs(level - want_level) < 1e-6, (p, exceeded, level, want_level)


def test_layers_errors():
    rows = np.zeros(1, dtype=abi.PERIOD_LINE_DTYPE)
    rows[0]["energy"], rows[0]["means"], rows[0]["lambda"] = 1.0, 1.0, math.inf
    rows[0]["duty"], rows[0]["passing"] = math.nan, math.nan
    bad = rows.copy()
    bad[0]["layer"] = 2
    for case, steady, words in ((bad, [0.0, 0.0], "names layer 2"), (rows, [-1.0], "steady energy of layer 0")):
        with pytest.raises(native.QmError) as err:
            native.distribution_layers(0.5, case, steady)
        assert err.value.status == abi.QM_ERR_ARGUMENT and words in str(err.value)
    for field, value in (("lambda", math.nan), ("duty", 1.5)):
        bad = rows.copy()
        bad[0][field] = value
        with pytest.raises(native.QmError) as err:
            native.distribution_layers(0.5, bad, [0.0])
        assert err.value.status == abi.QM_ERR_ARGUMENT and "line 0" in str(err.value)
    bad = rows.copy()
    bad[0]["means"][3] = -1.0
    with pytest.raises(native.QmError):
        native.distribution_layers(0.5, bad, [0.0])
    # A steady line alone holds its mean in every state: one bin, all the time.
    layer_bins, silent, place, place_silent = native.distribution_layers(0.5, rows, [0.0])
    assert silent[0] == 0.0 and np.count_nonzero(layer_bins[0][:, 0]) == 1
    assert abs(native.distribution_exceeded_db(0.5, place, 0.99)) < 1e-9 and place_silent == 0.0


@pytest.mark.parametrize("bin_db", [0.5, 2.0])
def test_profiled_roads_over_groups_of_hours_match_the_oracle(bin_db):
    """Roads that follow an hourly profile, over groups of a period's hours with their own flow
    factors (the map's four, one and three groups of 16, 4 and 8 hours), beside layers that follow
    none: every layer's and the place's distribution equal the oracle's to the bit. The dense
    roads' lambda drops under 10 in quiet groups, so their shape changes from group to group."""
    rng = np.random.default_rng(8)
    layers = _place(11, sparse=False)
    roads_index = 0
    road_lines = layers[roads_index][0]
    profiled_roads = [True, False]
    hours_of = [16, 4, 8]
    groups_of = [[4, 4, 4, 4], [4], [3, 3, 2]]
    groups = []
    factors_of = []
    for p in range(3):
        per_group = []
        factor_rows = []
        for slots in groups_of[p]:
            road_factors = [float(rng.uniform(0.2, 2.0)) if prof else 1.0 for prof in profiled_roads]
            per_layer = [road_factors if k == roads_index else None for k in range(len(layers))]
            per_group.append((slots, per_layer))
            factor_rows.append(road_factors + [1.0] * (sum(len(lines) for lines, _ in layers) - len(road_lines)))
        groups.append((hours_of[p], per_group))
        factors_of.append(factor_rows)
    each, whole = dist.layered_distributions(layers, bin_db, groups)
    profiled = profiled_roads + [False] * (sum(len(lines) for lines, _ in layers) - len(road_lines))
    for p in range(3):
        got_each, got_silent, got_whole, got_whole_silent = native.distribution_layers_grouped(
            bin_db, _period_rows(layers, p), [steady[p] for _, steady in layers], hours_of[p], groups_of[p],
            factors_of[p], profiled)
        for k in range(len(layers)):
            assert np.array_equal(got_each[k], _bins(each[k][p])) and got_silent[k] == each[k][p].silent, (p, k)
        assert np.array_equal(got_whole, _bins(whole[p])) and got_whole_silent == whole[p].silent, p
    with pytest.raises(native.QmError) as err:
        native.distribution_layers_grouped(bin_db, _period_rows(layers, 0), [s[0] for _, s in layers], 15,
                                           groups_of[0], factors_of[0], profiled)
    assert err.value.status == abi.QM_ERR_ARGUMENT and "16 hours" in str(err.value)


def _road_thirds():
    """A broadband spectrum peaking near 1 kHz, 2 dB down a band either side (energies)."""
    return [dist.energy(60.0 - 2.0 * abs(k - 16)) for k in range(28)]


def _of_levels(levels, bin_db=0.5):
    return dist.Distribution.of_levels(levels, bin_db)


def test_loudness_matches_the_oracle_and_counts_how_long_a_sound_lasts():
    """Mean loudness and Nden from the distributions equal the oracle's to the bit on the same
    curves; and as the reference's test states (popup/src/loudness.rs:396-424): a sound heard half
    of each period reads half its steady loudness; a pass loud a hundredth of the time adds a
    hundredth of its loudness; a sound in the day alone reads half its day in Nden, one at night
    alone a third of its loudness 10 dB up."""
    curve = dist.Curve(_road_thirds())
    shape = native.loudness_curve_shape(_road_thirds())
    assert np.array_equal(shape, np.array(curve.shape_db))
    assert native.loudness_curve_shape([0.0] * 28) is None
    curves = np.array([curve.table] * 3)

    def both(distributions):
        bins = np.array([_bins(d) for d in distributions])
        got_mean, got_nden = native.distribution_loudness(0.5, bins, curves)
        want_mean, want_nden = dist.loudness(distributions, [curve] * 3)
        assert np.array_equal(got_mean, np.array(want_mean)) and got_nden == want_nden
        return got_mean, got_nden

    silent = _of_levels([(-math.inf, 1.0)])
    steady, _ = both([_of_levels([(60.0, 1.0)])] * 3)
    half, _ = both([_of_levels([(60.0, 0.5), (-math.inf, 0.5)])] * 3)
    assert abs(half[0] / steady[0] - 0.5) < 1e-9
    rare, _ = both([_of_levels([(40.0, 0.99), (80.0, 0.01)])] * 3)
    expected = 0.99 * curve.at(40.0) + 0.01 * curve.at(80.0)
    assert abs(rare[0] - expected) < 1e-9 * expected
    day_mean, day_nden = both([_of_levels([(60.0, 1.0)]), silent, silent])
    assert abs(day_nden - day_mean[0] / 2.0) < 1e-9
    _, night_nden = both([silent, silent, _of_levels([(60.0, 1.0)])])
    assert abs(night_nden - curve.at(70.0) / 3.0) < 1e-9
    nothing, nothing_nden = both([silent] * 3)
    assert np.array_equal(nothing, np.zeros(3)) and nothing_nden == 0.0
    # A road-like sound's loudness about doubles per 10 dB (loudness.rs:351-391).
    assert 1.8 < curve.at(70.0) / curve.at(60.0) < 2.3 and 10.0 < curve.at(65.0) < 30.0


def test_loudness_of_a_place_matches_the_oracle():
    """The place of the layer tests, its three periods' distributions read on three curves."""
    layers = _place(7, sparse=False)
    _, whole = dist.layered_distributions(layers, 0.5)
    curves = [dist.Curve([dist.energy(55.0 + p * 3.0 - 1.5 * abs(k - 14 - p)) for k in range(28)]) for p in range(3)]
    bins = np.array([_bins(whole[p]) for p in range(3)])
    got_mean, got_nden = native.distribution_loudness(0.5, bins, np.array([c.table for c in curves]))
    want_mean, want_nden = dist.loudness(whole, curves)
    assert np.array_equal(got_mean, np.array(want_mean)) and got_nden == want_nden and got_nden > 0.0


def test_weather_state_means_match_the_oracle_to_the_bit():
    """Random pieces, some louder downwind, some in calm air, some without states, some silent in
    a period: a line's means in the weather states equal the oracle's to the bit, and their
    average is the line's energy where its pieces make it up."""
    rng = np.random.default_rng(31)
    for trial in range(300):
        n = int(rng.integers(0, 8))
        weather = dist.Weather()
        piece_energy, piece_states = [], []
        for _ in range(n):
            calm = 10.0 ** rng.uniform(0.0, 6.0, 3)
            favourable = calm * 10.0 ** rng.uniform(-1.0, 1.5, 3)
            share = rng.uniform(0.0, 1.0, 3)
            mean = calm + share * (favourable - calm)
            if rng.random() < 0.15:
                calm, favourable = np.zeros(3), np.zeros(3)
            if rng.random() < 0.1:
                mean[int(rng.integers(0, 3))] = 0.0
            weather.add(list(mean), [list(calm), list(favourable)])
            piece_energy.append(mean)
            piece_states.append([calm, favourable])
        energy = np.sum(piece_energy, axis=0) if n else 10.0 ** rng.uniform(0.0, 3.0, 3)
        want = dist.weather_means(weather, list(energy))
        got = native.distribution_state_means(np.array(piece_energy).reshape(-1, 3),
                                              np.array(piece_states).reshape(-1, 2, 3), energy)
        assert np.array_equal(got, np.array(want)), trial
    # Pieces louder in opposite states keep their mean (percentiles_tests.rs:283-306).
    pieces = [(1.0, 10.0, 0.41), (10.0, 1.0, 0.49)]
    means = [calm + share * (down - calm) for calm, down, share in pieces]
    got = native.distribution_state_means([[m] * 3 for m in means],
                                          [[[calm] * 3, [down] * 3] for calm, down, _ in pieces], [sum(means)] * 3)
    assert abs(got[0].mean() - sum(means)) < 1e-9


def test_a_pixel_from_its_pieces_to_nden_matches_the_oracle():
    """The chain a pixel's loudness takes, every step through the library and checked against the
    oracle: each line's means in the weather states from its pieces' calm and favourable
    energies, merged where close (the map's spread 1.2), the period's layers on the map's 2 dB grid
    (roads, bells, flights, steady energy), and each period's loudness on its curve and Nden."""
    rng = np.random.default_rng(41)
    states = dist.WEATHER_STATES
    layers_oracle = []
    for layer in range(3):
        lines = []
        for k in range(3):
            weather = dist.Weather()
            total = np.zeros(3)
            piece_energy, piece_states = [], []
            for _ in range(int(rng.integers(1, 4))):
                calm = 10.0 ** rng.uniform(2.0, 5.0, 3)
                favourable = calm * 10.0 ** rng.uniform(0.0, 1.0, 3)
                mean = calm + rng.uniform(0.0, 1.0, 3) * (favourable - calm)
                weather.add(list(mean), [list(calm), list(favourable)])
                piece_energy.append(mean)
                piece_states.append([calm, favourable])
                total += mean
            means = dist.weather_means(weather, list(total))
            assert np.array_equal(native.distribution_state_means(piece_energy, piece_states, total), means)
            if layer == 1 and k == 0:
                lines.append(dist.Line(list(total), means, [math.inf] * 3, duty=[0.05, 0.02, 0.0]))
            elif layer == 2:
                lines.append(dist.Line(list(total), means, [math.inf] * 3, passing=[0.05 * (k + 1), 0.1, 0.0]))
            else:
                lines.append(dist.Line(list(total), means, [40.0, 20.0, 12.0]))
        layers_oracle.append((lines, list(10.0 ** rng.uniform(1.0, 3.0, 3))))
    dist.merge_close_states(layers_oracle, 1.2)
    curves = [dist.Curve([dist.energy(58.0 - 1.8 * abs(k - 15 - p)) for k in range(28)]) for p in range(3)]
    each, whole = dist.layered_distributions(layers_oracle, 2.0)
    want_mean, want_nden = dist.loudness(whole, curves)

    bins = []
    for p in range(3):
        rows = _period_rows(layers_oracle, p)
        rows = native.distribution_merge_states(rows, 1.2)    # already merged: a fixed point
        assert np.array_equal(rows["means"], _period_rows(layers_oracle, p)["means"])
        layer_bins, layer_silent, place, place_silent = native.distribution_layers(
            2.0, rows, [steady[p] for _, steady in layers_oracle])
        assert np.array_equal(place, _bins(whole[p])) and place_silent == whole[p].silent
        bins.append(place)
    got_mean, got_nden = native.distribution_loudness(2.0, np.array(bins), np.array([c.table for c in curves]))
    assert np.array_equal(got_mean, np.array(want_mean)) and got_nden == want_nden and got_nden > 0.0


def test_hour_groups_match_the_oracle_and_feed_the_grouped_layers():
    """Over random hourly shares of three profiles: each period's hours, apart or in the map's
    four, one and three groups, and each profile's flow factor per group equal the oracle's to the
    bit; the groups cover the period's hours and a profile's factors average to 1 over them. A
    profiled road over those groups then gives the oracle's distributions to the bit."""
    rng = np.random.default_rng(17)
    shares = rng.uniform(0.3, 9.0, (3, 24))
    for period in range(3):
        hours = int(dist.PERIOD_HOURS[period])
        for runs in (0, 1, 2, [4, 1, 3][period], hours):
            slot_group, group_hours, factors = native.hour_groups(shares, period, runs)
            groups, want_hours = dist.hour_groups(shares.tolist(), period, runs or None)
            assert want_hours == hours and len(group_hours) == len(groups) and group_hours.sum() == hours
            for g, slots in enumerate(groups):
                assert group_hours[g] == len(slots) and all(slot_group[s] == g for s in slots)
                for profile in range(3):
                    assert factors[g, profile] == dist.group_factor(shares.tolist(), profile, period, slots)
            for profile in range(3):
                assert abs((factors[:, profile] * group_hours).sum() / hours - 1.0) < 1e-12
    with pytest.raises(native.QmError):
        native.hour_groups(shares, 1, 5)
    bad = shares.copy()
    bad[1, 3] = 0.0
    with pytest.raises(native.QmError):
        native.hour_groups(bad, 0, 4)

    # A profiled road (profile 1) beside a steady layer, over the map's groups.
    states = dist.WEATHER_STATES
    road = dist.Line([dist.energy(60.0)] * 3, [[dist.energy(60.0) * (1.0 + 0.05 * s) for s in range(states)]] * 3,
                     [30.0, 15.0, 11.0])
    layers = [([road], [0.0] * 3), ([], [dist.energy(45.0)] * 3)]
    oracle_groups = []
    for period in range(3):
        groups, hours = dist.hour_groups(shares.tolist(), period, [4, 1, 3][period])
        oracle_groups.append((hours, [(len(slots), [[dist.group_factor(shares.tolist(), 1, period, slots)], None])
                                      for slots in groups]))
    each, whole = dist.layered_distributions(layers, 2.0, oracle_groups)
    for period in range(3):
        _, group_hours, factors = native.hour_groups(shares, period, [4, 1, 3][period])
        got_each, _, got_whole, got_silent = native.distribution_layers_grouped(
            2.0, _period_rows(layers, period), [steady[period] for _, steady in layers],
            int(dist.PERIOD_HOURS[period]), group_hours, factors[:, [1]], [True])
        assert np.array_equal(got_whole, _bins(whole[period])) and got_silent == whole[period].silent
        assert np.array_equal(got_each[0], _bins(each[0][period]))


def test_percentiles_of_a_place():
    """Percentiles::of (popup/src/percentiles.rs:284-296): the place's levels exceeded 5, 10, 50
    and 90 % of each period, equal to the oracle's; a silent period reads -inf."""
    layers = _place(9, sparse=False)
    _, whole = dist.layered_distributions(layers, 0.5)
    bins = np.array([_bins(whole[p]) for p in range(3)])
    got = native.distribution_percentiles(0.5, bins)
    for k, exceeded in enumerate((0.05, 0.1, 0.5, 0.9)):
        for p in range(3):
            assert got[k, p] == whole[p].exceeded_db(exceeded)
    assert np.all(np.diff(got[:, 0]) <= 0.0), "L5 >= L10 >= L50 >= L90"
    silent = np.zeros((3, 360, 2))
    assert np.all(np.isneginf(native.distribution_percentiles(0.5, silent)))
