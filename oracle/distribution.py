"""How levels add over time (popup/src/distribution.rs), restated in Python — TEST INFRASTRUCTURE
ONLY.

A distribution of the summed level over a period on a grid of bin_db decibels from -30 dB over
180 dB: per bin its share of the time and that share times its moments' mean intensity, so that
adding an independent sound loses no energy to the grid; silence apart. A line's values are its
intensities relative to its mean at fixed probabilities with the share of the time each stands
for (Kurze's quantiles, `oracle.relative_intensity`), an event's mean over its duty, or a
Poisson stream of passes. Only tests import this module.
"""

import bisect
import math

from oracle import oracle

LEVEL_MIN_DB = -30.0   # distribution.rs:11
SPAN_DB = 180.0        # distribution.rs:12
LN_10 = 2.302585092994046


def energy(level_db):
    """physics/src/bands.rs:34-36."""
    return math.exp(level_db * (LN_10 / 10.0))


def _round_half_away(x):
    f = math.floor(x)
    return f + 1.0 if x - f >= 0.5 else f


def node_probabilities():
    """distribution.rs:17-32: every percent to 0.99, then evenly in log(1 - p) to 1 - 1e-8, each
    with the share of the time it stands for."""
    nodes = [((k + 0.5) / 100.0, 0.01) for k in range(99)]
    at = lambda t: 1.0 - 10.0 ** (-t)
    for k in range(24):
        a, b = 2.0 + k * 0.25, 2.25 + k * 0.25
        nodes.append((at((a + b) / 2.0), at(b) - at(a)))
    nodes.append((1.0 - 0.5e-8, 1e-8))
    return nodes


class LineValues:
    """Intensities with their shares of the time, ascending, and the running sums of the shares
    and of the shares times the intensities (distribution.rs:236-262)."""

    def __init__(self, pairs):
        self.pairs = sorted(((float(v), float(s)) for v, s in pairs), key=lambda p: p[0])
        self.values = [v for v, _ in self.pairs]
        self.sums = [(0.0, 0.0)]
        for value, share in self.pairs:
            shares, weighted = self.sums[-1]
            self.sums.append((shares + share, weighted + share * value))


def line_values(lam, duty=None):
    """distribution.rs:264-281: Kurze's quantiles at `lam` at the nodes, or an event's mean over
    its duty while it sounds and silence otherwise."""
    if duty is not None:
        return LineValues([(0.0, 1.0 - duty), (1.0 / duty, duty)])
    nodes = node_probabilities()
    values = oracle.relative_intensity(lam, [p for p, _ in nodes])
    return LineValues(list(zip(values, [s for _, s in nodes])))


def pass_values(mean):
    """distribution.rs:283-298: passes of one level, a Poisson number `mean` in progress on
    average, each at the stream's mean over `mean`; the numbers up to the one a moment in 1e12
    exceeds, which takes what is left of the time and of the mean."""
    share = math.exp(-mean)
    pairs = [(0.0, share)]
    time_left, mean_left = -math.expm1(-mean), 1.0
    count = 0.0
    while True:
        count += 1.0
        share *= mean / count
        if time_left - share <= 1e-12:
            pairs.append((mean_left / time_left, time_left))
            return LineValues(pairs)
        time_left -= share
        mean_left -= share * count / mean
        pairs.append((count / mean, share))


class Distribution:
    """distribution.rs:44-221."""

    def __init__(self, bin_db):
        self.silent = 0.0
        self.bin_db = bin_db
        self.bins = [[0.0, 0.0] for _ in range(int(_round_half_away(SPAN_DB / bin_db)))]

    def bin_count(self):
        return len(self.bins)

    def bin(self, level_db):
        """The bin of a level; one under the grid is held in its lowest bin (distribution.rs:69-73)."""
        x = (level_db - LEVEL_MIN_DB) / self.bin_db
        index = 0 if math.isnan(x) else max(_round_half_away(x), 0.0)
        return int(min(index, len(self.bins) - 1))

    def intensities(self):
        """Each bin holding time: its moments' mean intensity and its share."""
        return [(weighted / share, share) for share, weighted in self.bins if share > 0.0]

    def runs(self, intensity, line, scale, visit):
        """The bins a moment at `intensity` moves to with each of the line's values times `scale`
        added (`None`: silence), each visited once in increasing order with the shares of the
        values that take it there and their shares times their values (distribution.rs:91-145)."""
        pairs, sums, values = line.pairs, line.sums, line.values

        def run(a, b):
            return (sums[b][0] - sums[a][0], scale * (sums[b][1] - sums[a][1]))

        start = 0
        if intensity <= 0.0:
            start = bisect.bisect_right(values, 0.0)
            if start > 0:
                visit(None, run(0, start))
        if start == len(pairs):
            return
        last = len(self.bins) - 1
        step = energy(self.bin_db)
        b = self.bin(10.0 * math.log10(intensity + scale * pairs[start][0]))
        ceiling = energy(LEVEL_MIN_DB + (b + 0.5) * self.bin_db)
        while True:
            if b == last:
                to = len(pairs)
            else:
                to = bisect.bisect_left(values, (ceiling - intensity) / scale, start + 1)
            visit(b, run(start, to))
            start = to
            if start >= len(pairs):
                break
            value = pairs[start][0]
            while True:
                b += 1
                ceiling *= step
                if b == last or intensity + scale * value < ceiling:
                    break

    def exceeded_db(self, exceeded):
        """The level exceeded `exceeded` of the time (distribution.rs:152-162)."""
        above = 0.0
        for share, weighted in reversed(self.bins):
            above += share
            if share > 0.0 and above > exceeded * (1.0 - 1e-12):
                return 10.0 * math.log10(weighted / share)
        return -math.inf

    def with_line(self, line, scale=1.0):
        """This distribution with an independent line (values times `scale`) added at every moment
        (distribution.rs:176-196)."""
        out = Distribution(self.bin_db)

        def add(intensity, share):
            def visit(b, sums):
                shares, weighted = sums
                if b is None:
                    out.silent += share * shares
                else:
                    out.bins[b][0] += share * shares
                    out.bins[b][1] += share * (intensity * shares + weighted)
            self.runs(intensity, line, scale, visit)

        if self.silent > 0.0:
            add(0.0, self.silent)
        for intensity, share in self.intensities():
            add(intensity, share)
        return out

    def with_distribution(self, other):
        """This with an independent `other` added: its levels as a line's values, its silence a
        value of nothing (distribution.rs:198-206)."""
        values = [(i, s) for i, s in other.intensities()] + [(0.0, other.silent)]
        return self.with_line(LineValues([(i, s) for i, s in values if s > 0.0]))

    def over(self, intensity):
        """With a steady intensity added at every moment."""
        return self.with_line(LineValues([(intensity, 1.0)]))

    def add_scaled(self, other, weight):
        self.silent += other.silent * weight
        for into, source in zip(self.bins, other.bins):
            into[0] += source[0] * weight
            into[1] += source[1] * weight

    @staticmethod
    def of_levels(levels, bin_db=0.5):
        """A distribution of given levels (dB, -inf silent) with their shares of the time."""
        silence = Distribution(bin_db)
        silence.silent = 1.0
        return silence.with_line(LineValues([(10.0 ** (level / 10.0), share) for level, share in levels]))


# ---------------------------------------------------------------------------------------------
# Layers of lines over a period (popup/src/percentiles.rs:88-282, percentiles/lines.rs:8-248),
# without hourly profiles: every line at its period's mean flow, one group of hours.

WEATHER_STATES = 10                      # percentiles/weather.rs:131
HOLDS_MEAN_LAMBDA = 10.0                 # lines.rs:240
PASSES_HOLD_MEAN = 2.0 * math.pi * HOLDS_MEAN_LAMBDA   # lines.rs:243
HELD_EXCEEDED = 1e-3                     # lines.rs:247
HELD_SHARE = 1e-2                        # lines.rs:248
MIN_POSITIVE = 2.2250738585072014e-308   # the least normal f64


class Line:
    """One source whose level varies in time, per period (lines.rs:8-24): its mean energy, its
    means in the weather states, Kurze's lambda, an event's duty or a stream's passes in
    progress (None: not that kind)."""

    def __init__(self, energy, means, lam, duty=None, passing=None):
        self.energy = list(energy)
        self.means = [list(m) for m in means]
        self.lam = list(lam)
        self.duty = None if duty is None else list(duty)
        self.passing = None if passing is None else list(passing)

    def shape(self, period, factor=1.0):
        """(values, exceeded) where the line moves the level in `period`, None where it holds
        its mean or is silent (lines.rs:172-195): a stream's passes unless that many hold the
        mean, an event's duty while it sounds, a sparse line's Kurze values with the intensity
        it exceeds a thousandth of the time."""
        if self.passing is not None:
            mean = self.passing[period]
            return (pass_values(mean), None) if MIN_POSITIVE <= mean < PASSES_HOLD_MEAN else None
        lam = self.lam[period] * factor
        if self.duty is not None:
            duty = self.duty[period]
            return (line_values(0.0, duty=duty), None) if duty > 0.0 else None
        if lam >= HOLDS_MEAN_LAMBDA:
            return None
        return line_values(lam), oracle.relative_intensity(lam, 1.0 - HELD_EXCEEDED)


def moment(lines, shapes, state_means, factors, steady, period):
    """The energy that holds steady and the lines that move the level (percentiles.rs:236-282):
    (floor, holding [(index, mean)], moving [(index, values, mean)]), the events and streams
    first, then the sparse lines whose level exceeded a thousandth of the time reaches a
    hundredth of the steady energy."""
    floor, holding, moving, held = steady, [], [], []
    for index, (line, shape) in enumerate(zip(lines, shapes)):
        mean = state_means[index] * factors[index]
        if line.energy[period] <= 0.0 or mean <= 0.0:
            continue
        if shape is not None and shape[1] is None:
            moving.append((index, shape[0], mean))
        elif shape is not None:
            held.append((index, shape[0], mean, shape[1]))
        elif line.duty is not None:
            continue
        else:
            floor += mean
            holding.append((index, mean))
    # The held lines' means summed on their own, then added to the floor (percentiles.rs:270-272).
    steady_energy = floor + sum(mean for _, _, mean, _ in held)
    for index, values, mean, exceeded in held:
        if mean * exceeded < HELD_SHARE * steady_energy:
            floor += mean
            holding.append((index, mean))
        else:
            moving.append((index, values, mean))
    return floor, holding, moving


def layer_states(lines, steady, period, bin_db, factors=None):
    """A layer's distribution in each weather state of `period` with its floor where no line
    moves (percentiles.rs:172-211): its steady energy and holding lines first, then each moving
    line added. `factors`: each line's flow in the hours against the period's mean (1 without a
    profile)."""
    factors = [1.0] * len(lines) if factors is None else list(factors)
    shapes = [line.shape(period, factor) for line, factor in zip(lines, factors)]
    states = []
    for state in range(WEATHER_STATES):
        if state > 0 and all(line.means[period][state] == line.means[period][state - 1] for line in lines):
            states.append(states[-1])
            continue
        state_means = [line.means[period][state] for line in lines]
        floor, _, moving = moment(lines, shapes, state_means, factors, steady, period)
        total = Distribution(bin_db)
        total.silent = 1.0
        total = total.over(floor)
        for _, values, mean in moving:
            total = total.with_line(values, mean)
        states.append((total, floor if not moving else None))
    return states


def layered_distributions(layers, bin_db, groups=None):
    """Per period each layer's distribution and the place's (percentiles.rs:88-160) for layers of
    (lines, steady per period): for every group of hours and weather state, each layer's
    distribution, and the place's with the steady layers' floors summed and the moving layers'
    distributions added as independent sounds; the groups and states averaged by their shares of
    the time. `groups` (None: no line follows a profile) gives per period (hours, [(hours in the
    group, per layer its lines' flow factors in the group or None where no line of the layer
    follows a profile)]); a layer with no profiled line is computed once at its mean flow."""
    each = [[None] * 3 for _ in layers]
    whole = []
    for p in range(3):
        hours, parts_of = (1, [(1, [None] * len(layers))]) if groups is None else groups[p]
        alike = [layer_states(lines, steady[p], p, bin_db) if parts_of[0][1][k] is None else None
                 for k, (lines, steady) in enumerate(layers)]
        parts = []
        for slots, factors in parts_of:
            own = [None if alike[k] is not None else layer_states(lines, steady[p], p, bin_db, factors[k])
                   for k, (lines, steady) in enumerate(layers)]
            wholes = []
            for state in range(WEATHER_STATES):
                states = [(own[k] if own[k] is not None else alike[k])[state] for k in range(len(layers))]
                floor = 0.0
                for _, f in states:
                    if f is not None:
                        floor += f
                total = Distribution(bin_db)
                total.silent = 1.0
                total = total.over(floor)
                for part, f in states:
                    if f is None:
                        total = total.with_distribution(part)
                wholes.append(total)
            parts.append((slots / (hours * WEATHER_STATES), own, wholes))
        mixtures = []
        for k in range(len(layers)):
            mixture = Distribution(bin_db)
            if alike[k] is not None:
                for part, _ in alike[k]:
                    mixture.add_scaled(part, 1.0 / WEATHER_STATES)
            mixtures.append(mixture)
        mixed = Distribution(bin_db)
        for weight, own, wholes in parts:
            for k in range(len(layers)):
                if own[k] is not None:
                    for part, _ in own[k]:
                        mixtures[k].add_scaled(part, weight)
            for part in wholes:
                mixed.add_scaled(part, weight)
        for k in range(len(layers)):
            each[k][p] = mixtures[k]
        whole.append(mixed)
    return each, whole


def merge_close_states(layers, spread):
    """The weather states merged where their difference cannot show (percentiles/weather.rs:
    132-176): per period, each run of consecutive states in which every line's mean is finite and
    within `spread` (largest over smallest) gives each line its mean over the run in all of the
    run's states. Changes the lines' means in place."""
    def within(means):
        low, high = math.inf, 0.0
        for mean in means:
            if not math.isfinite(mean):
                return False
            low, high = min(low, mean), max(high, mean)
        return high <= spread * low

    lines = [line for layer_lines, _ in layers for line in layer_lines]
    for period in range(3):
        start = 0
        while start < WEATHER_STATES:
            end = start + 1
            while end < WEATHER_STATES and all(within(line.means[period][start:end + 1]) for line in lines):
                end += 1
            if end - start > 1:
                for line in lines:
                    run = line.means[period][start:end]
                    if any(mean != run[0] for mean in run):
                        total = 0.0
                        for mean in run:
                            total += mean
                        line.means[period][start:end] = [total / len(run)] * len(run)
            start = end


# ---------------------------------------------------------------------------------------------
# Loudness from the distributions (popup/src/loudness.rs:68-130, 236-269).

CURVE_LOW_DB, CURVE_HIGH_DB = -30.0, 160.0          # loudness.rs:68-69
PERIOD_HOURS = (12.0, 4.0, 8.0)                     # physics/src/bands.rs:16
PERIOD_PENALTY_DB = (0.0, 5.0, 10.0)                # physics/src/bands.rs:18
# Third-octave A-weighting, 25 Hz to 12.5 kHz (IEC 61672-1; physics/src/loudness.rs:14-17).
A_WEIGHTING_THIRDS_DB = (-44.7, -39.4, -34.6, -30.2, -26.2, -22.5, -19.1, -16.1, -13.4, -10.9, -8.6, -6.6,
                         -4.8, -3.2, -1.9, -0.8, 0.0, 0.6, 1.0, 1.2, 1.3, 1.2, 1.0, 0.5, -0.1, -1.1, -2.5, -4.3)


class Curve:
    """One period's loudness by A-weighted level (loudness.rs:74-130): the received spectrum (28
    third-octave energies) set to each whole decibel from -30 to 160 dB, Zwicker's loudness there,
    linear between."""

    def __init__(self, thirds):
        a_weighted = 0.0
        for value, weight in zip(thirds, A_WEIGHTING_THIRDS_DB):
            a_weighted += value * energy(weight)
        self.shape_db = None
        if a_weighted > 0.0:
            self.shape_db = [10.0 * math.log10(v / a_weighted) if v > 0.0 else -math.inf for v in thirds]
        steps = int(CURVE_HIGH_DB - CURVE_LOW_DB)
        if self.shape_db is None:
            self.table = [0.0] * (steps + 1)
        else:
            self.table = list(oracle.zwicker_many([[db + (CURVE_LOW_DB + step) for db in self.shape_db]
                                                   for step in range(steps + 1)]))

    def at(self, level_db):
        last = int(CURVE_HIGH_DB - CURVE_LOW_DB)
        position = min(max(level_db - CURVE_LOW_DB, 0.0), float(last))
        below = min(int(math.floor(position)), last - 1)
        low, high = self.table[below], self.table[below + 1]
        return low + (high - low) * (position - below)


def loudness(distributions, curves):
    """Each period's mean loudness and Nden (loudness.rs:236-269): per period the levels' shares
    times the curve there (the evening's 5 dB and the night's 10 dB added for Nden), the periods
    over their hours."""
    def mean(penalty):
        out = []
        for p in range(3):
            total = 0.0
            for intensity, share in distributions[p].intensities():
                total += share * curves[p].at(10.0 * math.log10(intensity) + penalty(p))
            out.append(total)
        return out

    mean_sone = mean(lambda p: 0.0)
    penalised = mean(lambda p: PERIOD_PENALTY_DB[p])
    day = 0.0
    for p in range(3):
        day += PERIOD_HOURS[p] * penalised[p]
    return mean_sone, day / 24.0


# ---------------------------------------------------------------------------------------------
# A line's means in the weather states from its pieces' energies in the two meteorological states
# (popup/src/percentiles/weather.rs:1-127).

SHARE_BINS = 10                          # weather.rs:6
EPSILON = 2.220446049250313e-16          # f64::EPSILON


def favourable_share(mean, homogeneous, favourable):
    """The share of the time in the favourable state, from the mean being the mix of the two
    (weather.rs:77-84)."""
    if abs(favourable - homogeneous) <= EPSILON * abs(favourable):
        return 0.0
    return min(max((mean - homogeneous) / (favourable - homogeneous), 0.0), 1.0)


class Weather:
    """A contributor's energy per period in each state (homogeneous, favourable) and mixed, binned
    by its pieces' favourable share, pieces louder in calm air in bins of their own
    (weather.rs:7-75)."""

    def __init__(self):
        self.bins = [[[0.0] * 3 for _ in range(3)] for _ in range(2 * SHARE_BINS)]
        self.active = 0

    @staticmethod
    def binned(energy, states):
        homogeneous, favourable = states if (states[0] > 0.0 or states[1] > 0.0) else (energy, energy)
        share = favourable_share(energy, homogeneous, favourable)
        calm_louder = 1 if favourable < homogeneous else 0
        position = share * SHARE_BINS
        bin_ = calm_louder * SHARE_BINS + min(int(position) if position == position else 0, SHARE_BINS - 1)
        return bin_, (homogeneous, favourable, energy)

    def add_binned(self, period, bin_, values):
        self.active |= 1 << bin_
        for state, value in enumerate(values):
            self.bins[bin_][state][period] += value

    def add(self, energy, states):
        """A piece of `energy` per period, the mix of its states[0] (homogeneous) and states[1]
        (favourable) per period."""
        for period in range(3):
            bin_, values = Weather.binned(energy[period], (states[0][period], states[1][period]))
            self.add_binned(period, bin_, values)


def weather_means(weather, energy):
    """Per period the mean of `energy` in each weather state (weather.rs:85-127): each bin's calm
    energy in every state, its excess downwind in the states wholly under its share and in part
    in the state its share falls in."""
    if weather.active == 0:
        return [[energy[p]] * WEATHER_STATES for p in range(3)]
    out = []
    for period in range(3):
        whole, part = [0.0] * (WEATHER_STATES + 1), [0.0] * (WEATHER_STATES + 1)
        calm, silent = 0.0, True
        for bin_ in range(2 * SHARE_BINS):
            if not (weather.active >> bin_) & 1:
                continue
            homogeneous = weather.bins[bin_][0][period]
            favourable = weather.bins[bin_][1][period]
            mix = weather.bins[bin_][2][period]
            silent = silent and homogeneous + favourable <= 0.0
            share = favourable_share(mix, homogeneous, favourable)
            position = share * WEATHER_STATES
            state = min(int(position) if position == position else 0, WEATHER_STATES)
            whole[state] += favourable - homogeneous
            part[state] += (position - state) * (favourable - homogeneous)
            calm += homogeneous
        if silent:
            out.append([energy[period]] * WEATHER_STATES)
            continue
        means = [0.0] * WEATHER_STATES
        above = 0.0
        for state in reversed(range(WEATHER_STATES)):
            above += whole[state + 1]
            means[state] = calm + above + part[state]
        out.append(means)
    return out


# ---------------------------------------------------------------------------------------------
# Hours of a period grouped by their flow (popup/src/percentiles/traffic.rs:31-39, 251-279), over
# a caller's hourly shares per profile (shares[profile][24], by hour of the day).

PERIOD_FIRST_HOUR = (7, 19, 23)                     # traffic.rs:31


def hour_factor(shares, profile, period, slot):
    """A road's flow in the slot-th hour of the period against its mean over the period."""
    hours = int(PERIOD_HOURS[period])
    share = lambda s: shares[profile][(PERIOD_FIRST_HOUR[period] + s) % 24]
    total = 0.0
    for s in range(hours):
        total += share(s)
    return share(slot) / (total / hours)


def hour_groups(shares, period, runs):
    """(groups of slots, hours): every hour apart without `runs`, else the hours sorted by their
    flow summed over the profiles (ties by hour) cut into `runs` runs, each in hour order."""
    hours = int(PERIOD_HOURS[period])
    if runs is None:
        return [[slot] for slot in range(hours)], hours

    def flow(slot):
        total = 0.0
        for profile in range(len(shares)):
            total += hour_factor(shares, profile, period, slot)
        return total

    slots = sorted(range(hours), key=lambda slot: (flow(slot), slot))
    return [sorted(slots[run * hours // runs:(run + 1) * hours // runs]) for run in range(runs)], hours


def group_factor(shares, profile, period, slots):
    """A profiled line's flow over a group of hours: the mean of its hours' factors."""
    total = 0.0
    for slot in slots:
        total += hour_factor(shares, profile, period, slot)
    return total / len(slots)
