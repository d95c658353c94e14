"""Layers of lines over a period (popup/src/percentiles.rs:88-282 with percentiles/lines.rs),
restated in the oracle without hourly profiles, pinned to what the reference's tests state for
such places (popup/src/percentiles_tests.rs): bells ringing 2 % of the day beside a steady plant
(:372-416), flights heard while they pass beside it, a class of many passes holding its mean and
a faint class silent between its passes beside a loud one (:418-462); and the mixture's energy:
every layer's and the place's mean intensity is its lines' and steady energy's."""

import math

from oracle import distribution as dist

BIN_DB = 0.5  # the click's grid


def e(level_db):
    return dist.energy(level_db)


def steady_layer(level_db):
    return [], [e(level_db)] * 3


def flights(classes):
    """One flight line per class of (passes in progress by day, level dB): its energy that
    level by day and nothing otherwise, the same in every weather state."""
    lines = []
    for passing, level in classes:
        energy = [e(level), 0.0, 0.0]
        lines.append(dist.Line(energy, [[x] * dist.WEATHER_STATES for x in energy], [math.inf] * 3,
                               passing=[passing, 0.0, 0.0]))
    return lines, [0.0] * 3


def day_of(layers):
    return dist.layered_distributions(layers, BIN_DB)[1][0]


def mean_db(d):
    return 10.0 * math.log10(sum(share * e(level) for level, share in
                                 ((10.0 * math.log10(i), s) for i, s in d.intensities())))


def test_bells_sound_for_their_duty_and_are_silent_otherwise():
    bells = dist.Line([e(40.0)] * 3, [[e(40.0)] * dist.WEATHER_STATES] * 3, [math.inf] * 3,
                      duty=[0.02, 0.0, 0.01])
    day = day_of([steady_layer(40.0), ([bells], [0.0] * 3)])
    for exceeded in (0.05, 0.5, 0.9):
        assert abs(day.exceeded_db(exceeded) - 40.0) < 1e-9
    ringing = 10.0 * math.log10(51.0) + 40.0
    assert abs(day.exceeded_db(0.019) - ringing) <= BIN_DB / 2.0
    evening = dist.layered_distributions([steady_layer(40.0), ([bells], [0.0] * 3)], BIN_DB)[1][1]
    assert abs(evening.exceeded_db(0.001) - 40.0) < 1e-9, "an event off for the period is silent"


def test_flights_are_heard_while_they_pass():
    rare = day_of([steady_layer(40.0), flights([(0.02, 40.0)])])
    assert abs(rare.exceeded_db(0.015) - (10.0 * math.log10(51.0) + 40.0)) <= BIN_DB / 2.0
    assert abs(rare.exceeded_db(0.05) - 40.0) < 1e-9 and abs(rare.exceeded_db(0.9) - 40.0) < 1e-9
    often = day_of([steady_layer(40.0), flights([(0.2, 40.0)])])
    assert abs(often.exceeded_db(0.1) - (10.0 * math.log10(6.0) + 40.0)) <= BIN_DB / 2.0
    for d in (rare, often):
        assert abs(mean_db(d) - 10.0 * math.log10(2.0 * e(40.0))) < 1e-6
    dense = day_of([steady_layer(40.0), flights([(80.0, 40.0)])])
    whole = 10.0 * math.log10(2.0 * e(40.0))
    assert abs(dense.exceeded_db(0.01) - whole) < 1e-9 and abs(dense.exceeded_db(0.99) - whole) < 1e-9
    two = day_of([steady_layer(30.0), flights([(0.01, 35.0), (0.01, 80.0)])])
    for exceeded in (0.5, 0.9):
        assert abs(two.exceeded_db(exceeded) - 30.0) < 1e-9
    assert abs(two.exceeded_db(0.015) - 55.0) <= BIN_DB


def test_layers_keep_their_energy_in_every_weather_state():
    """Roads as sparse and dense Kurze lines whose means differ by weather state, events and
    passes in three layers over steady energy: each layer's mixture and the place's carry the
    mean of their parts' energies, period by period (the grid keeps intensities exact). A line
    that moves the level carries its mean times its values' own mean (a sparse line's Kurze
    values, read at the nodes up to 1 - 1e-8, carry their mean only to about 0.2 %, as in the
    reference's own energy test, distribution.rs:340-361); one that holds, its mean."""
    states = dist.WEATHER_STATES
    road = lambda base, lam: dist.Line([base] * 3, [[base * (1.0 + 0.1 * s) for s in range(states)]] * 3,
                                       [lam, lam * 0.5, lam * 0.2])
    roads = ([road(e(50.0), 0.03), road(e(45.0), 2.0), road(e(60.0), 40.0), road(e(20.0), 0.5)], [e(30.0)] * 3)
    bells = dist.Line([e(55.0)] * 3, [[e(55.0)] * states] * 3, [math.inf] * 3, duty=[0.05, 0.02, 0.0])
    events = ([bells], [0.0] * 3)
    planes = flights([(0.3, 50.0), (3.0, 45.0)])
    layers = [roads, events, planes]
    each, whole = dist.layered_distributions(layers, BIN_DB)

    def mean(d):
        return sum(i * s for i, s in d.intensities())

    moved = held = 0
    for p in range(3):
        expected = []
        for lines, steady in layers:
            shapes = [line.shape(p) for line in lines]
            total = 0.0
            for state in range(states):
                means = [line.means[p][state] for line in lines]
                floor, _, moving = dist.moment(lines, shapes, means, [1.0] * len(lines), steady[p], p)
                total += floor + sum(m * sum(v * w for v, w in values.pairs) for _, values, m in moving)
                moved += len(moving)
                held += len(lines) - len(moving)
            expected.append(total / states)
        for k in range(len(layers)):
            # A layer silent for the period (an event off, flights by day only) carries nothing.
            assert abs(mean(each[k][p]) - expected[k]) <= 1e-9 * expected[k], (p, k)
        assert abs(mean(whole[p]) - sum(expected)) <= 1e-9 * sum(expected), p
        assert abs(sum(s for _, s in whole[p].intensities()) + whole[p].silent - 1.0) < 1e-12
    assert moved > 50 and held > 50


def _line_of(means):
    states = dist.WEATHER_STATES
    return dist.Line([sum(means) / states] * 3, [list(means) for _ in range(3)], [1e6] * 3)


def test_close_weather_states_merge_and_keep_their_energy():
    """What the reference's test states (popup/src/percentiles_tests.rs:464-504): a line apart by
    more than the spread splits the states where it jumps; the other's first three states take
    their mean, the rest keep theirs; every line keeps its energy; means falling by more than the
    spread from state to state merge nowhere."""
    near = _line_of([1.10, 1.05, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    far = _line_of([4.0, 4.0, 4.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])
    before_near, before_far = list(near.means[0]), list(far.means[0])
    layers = [([near], [0.0] * 3), ([far], [0.0] * 3)]
    dist.merge_close_states(layers, 1.2)
    assert far.means[0] == before_far
    assert near.means[0][0] == near.means[0][2]
    assert abs(near.means[0][0] - (1.10 + 1.05 + 1.0) / 3.0) < 1e-12
    assert near.means[0][3:] == before_near[3:]
    for line in (near, far):
        assert abs(sum(line.means[0]) / dist.WEATHER_STATES - line.energy[0]) < 1e-12
    apart = _line_of([2.0, 1.5, 1.0, 0.7, 0.5, 0.35, 0.25, 0.18, 0.12, 0.09])
    before = [list(m) for m in apart.means]
    dist.merge_close_states([([apart], [0.0] * 3)], 1.2)
    assert apart.means == before


def test_the_library_merges_states_as_the_oracle_does():
    import numpy as np

    from quietmap_b200 import abi, native

    rng = np.random.default_rng(12)
    for trial in range(200):
        n = int(rng.integers(1, 6))
        lines = []
        for _ in range(n):
            base = 10.0 ** rng.uniform(-2.0, 6.0)
            steps = rng.choice([1.0, 1.0, 1.05, 1.15, 1.3, 3.0], size=dist.WEATHER_STATES)
            means = list(base * np.cumprod(steps) / steps[0])
            if trial % 17 == 0:
                means[int(rng.integers(0, dist.WEATHER_STATES))] = math.inf
            lines.append(_line_of(means))
        rows = np.zeros(n, dtype=abi.PERIOD_LINE_DTYPE)
        for k, line in enumerate(lines):
            rows[k]["means"] = line.means[0]
        spread = float(rng.choice([1.05, 1.2, 2.0]))
        merged = native.distribution_merge_states(rows, spread)
        dist.merge_close_states([(lines, [0.0] * 3)], spread)
        for k, line in enumerate(lines):
            assert np.array_equal(merged[k]["means"], np.array(line.means[0])), (trial, k)


def _steady_site(pieces, total=None):
    """A steady source made of pieces (energy, calm, favourable), the same every period: its line
    with means in the weather states."""
    weather = dist.Weather()
    energy = 0.0
    for mean, calm, favourable in pieces:
        weather.add([mean] * 3, [[calm] * 3, [favourable] * 3])
        energy += mean
    energy = energy if total is None else total
    return dist.Line([energy] * 3, dist.weather_means(weather, [energy] * 3), [math.inf] * 3)


def test_pieces_on_either_side_keep_their_own_weather():
    """percentiles_tests.rs:253-282: one piece always favourable (10 over calm 1), the other
    never: the level holds at their sum."""
    site = _steady_site([(10.0, 1.0, 10.0), (1.0, 1.0, 10.0)], total=11.0)
    day = dist.layered_distributions([([site], [0.0] * 3)], BIN_DB)[1]
    for p in range(3):
        for exceeded in (0.05, 0.5, 0.9):
            assert abs(day[p].exceeded_db(exceeded) - 10.0 * math.log10(11.0)) <= BIN_DB / 2.0


def test_pieces_louder_in_opposite_states_keep_their_mean():
    """percentiles_tests.rs:283-306: one piece louder downwind, one in calm air, in one share bin:
    the states average to the mean."""
    pieces, total = [], 0.0
    for calm, downwind, share in ((1.0, 10.0, 0.41), (10.0, 1.0, 0.49)):
        mean = calm + share * (downwind - calm)
        pieces.append((mean, calm, downwind))
        total += mean
    line = _steady_site(pieces)
    assert abs(sum(line.means[0]) / dist.WEATHER_STATES - total) < 1e-9


def test_a_source_alone_keeps_its_weather():
    """percentiles_tests.rs:307-338: favourable (50 dB) half the time and calm (40 dB) the other
    half, the source is at each for half the period."""
    calm, favourable = e(40.0), e(50.0)
    site = _steady_site([(0.5 * (calm + favourable), calm, favourable)])
    day = dist.layered_distributions([([site], [0.0] * 3)], BIN_DB)[1][0]
    levels = [(10.0 * math.log10(i), s) for i, s in day.intensities()]
    at = lambda db: sum(s for level, s in levels if abs(level - db) < 1e-9)
    assert abs(at(40.0) - 0.5) < 1e-9 and abs(at(50.0) - 0.5) < 1e-9, levels


def test_the_weather_moves_the_levels_smoothly():
    """percentiles_tests.rs:339-370: favourable 24.9 % and 25.1 % of the time (10 over calm 1)
    give nearly the same spread."""
    def spread(share):
        mean = share * 10.0 + (1.0 - share) * 1.0
        site = _steady_site([(mean, 1.0, 10.0)])
        return dist.layered_distributions([([site], [0.0] * 3)], BIN_DB)[1][0]

    below, above = spread(0.249), spread(0.251)
    mean = lambda d: sum(i * s for i, s in d.intensities())
    assert abs(mean(above) / mean(below) - 1.0) < 0.01
    for exceeded in (0.1, 0.5, 0.9):
        assert abs(above.exceeded_db(exceeded) - below.exceeded_db(exceeded)) < 0.2
