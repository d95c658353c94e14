"""No path gains more over free field from ground and diffraction than the relevance bound's
state maxima: the oracle's A_boundary pinned to the reference's own searched extremes and sampled
paths (physics/src/cnossos/boundary_gain_tests.rs), and a sliver of soft ground reading as hard
(physics/src/cnossos/ground.rs:147-170)."""

import numpy as np

from oracle import oracle

HOM, FAV = 0, 1
FAVOURABLE_GAIN_BOUND_DB = 18.0        # physics/src/bound.rs:12
HOMOGENEOUS_GAIN_BOUND_DB = 18.0       # physics/src/bound.rs:20
FLAT_HOMOGENEOUS_GAIN_BOUND_DB = 3.8   # boundary_gain_tests.rs:8
FLAT_FAVOURABLE_GAIN_BOUND_DB = 9.6    # boundary_gain_tests.rs:12


def gains(distance, altitude, ground, source, receiver, source_gf, terrain=(), tops=()):
    """Largest -A_boundary over the bands, per state."""
    att, _ = oracle.state_boundaries(distance, altitude, ground, source, receiver, source_gf,
                                     np.asarray(terrain, dtype=np.float64).reshape(-1, 2),
                                     np.asarray(tops, dtype=np.float64).reshape(-1, 2))
    return float(np.max(-att[HOM])), float(np.max(-att[FAV]))


def flat(length, source_z, receiver_z, tops=()):
    return gains([0.0, length], [0.0, 0.0], [0.0, 0.0], (0.0, source_z), (length, receiver_z), 0.0, (), tops)


def test_the_searched_extremes_stay_under_the_bound():
    assert 9.4 <= flat(10_000.0, 0.05, 4.0, [(9_900.0, 8.96)])[FAV] <= FLAT_FAVOURABLE_GAIN_BOUND_DB
    assert 3.5 <= flat(20_000.0, 0.05, 4.0, [(19_000.0, 1.80)])[HOM] <= FLAT_HOMOGENEOUS_GAIN_BOUND_DB
    assert 8.8 <= flat(29_000.0, 0.05, 4.0)[FAV] <= FLAT_FAVOURABLE_GAIN_BOUND_DB
    d, z = [0.0, 236.0, 11_800.0], [0.0, 14.57, 0.0]
    relief = gains(d, z, [0.0] * 3, (0.0, 0.05), (11_800.0, 1.5), 0.0, list(zip(d, z)))[FAV]
    assert 12.9 <= relief <= 13.3, relief


def test_below_plane_corners_stay_under_the_state_bounds():
    d = [0.0, 1325.533, 3827.411, 4293.855, 6218.238]
    z = [-85.685, -7.088, 28.333, 12.712, -44.696]
    fav = gains(d, z, [0.0, 0.0, 0.0, 0.0, 0.146], (0.0, -85.685 + 0.228), (6218.238, -44.696 + 7.241), 0.0,
                list(zip(d, z)))[FAV]
    assert 17.4 <= fav <= FAVOURABLE_GAIN_BOUND_DB, fav
    d = [0.0, 2003.806, 3406.244, 3462.741, 4428.192, 4645.091, 4888.823, 5042.429, 7571.335]
    z = [123.543, 105.373, -146.72, 13.508, -72.448, -52.391, 25.951, 72.715, 102.924]
    g = [0.0, 0.0, 0.004, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0]
    tops = [(743.466, 124.829), (2706.498, 123.986), (3843.265, 14.608)]
    hom = gains(d, z, g, (0.0, 123.543 + 1.814), (7571.335, 102.924 + 7.67), 0.0, list(zip(d, z)), tops)[HOM]
    assert 5.8 <= hom <= HOMOGENEOUS_GAIN_BOUND_DB, hom


class Samples:
    """The test's xorshift64* sequence (boundary_gain_tests.rs:176-192)."""

    def __init__(self, seed):
        self.s = seed

    def unit(self):
        mask = (1 << 64) - 1
        self.s ^= self.s >> 12
        self.s ^= (self.s << 25) & mask
        self.s ^= self.s >> 27
        return (((self.s * 0x2545_F491_4F6C_DD1D) & mask) >> 11) / float(1 << 53)

    def between(self, lo, hi):
        return lo + (hi - lo) * self.unit()

    def ground(self):
        return 0.0 if self.unit() < 0.4 else self.unit()


def test_no_sampled_path_gains_more_than_the_bound():
    """boundary_gain_tests.rs:199-309: 10,000 flat and 20,000 relief paths."""
    s = Samples(0x9E37_79B9_7F4A_7C15)
    worst = {"flat": [-np.inf, -np.inf], "relief": [-np.inf, -np.inf]}
    for sample in range(30_000):
        relief = sample >= 10_000
        length = 10.0 ** s.between(2.5 if relief else 0.7, 4.08)
        vertices = 2 + int(s.unit() * 8.0)
        distance = [s.between(0.0, length) for _ in range(vertices)]
        distance[0], distance[-1] = 0.0, length
        distance.sort()
        crest = relief and s.unit() < 0.5
        crest_x = s.between(0.05, 0.95) * length
        crest_h = s.between(1.0, 30.0)
        altitude = []
        for x in distance:
            if crest:
                altitude.append(crest_h * max(1.0 - abs((x - crest_x) / (0.5 * length)), 0.0)
                                + s.between(-0.005, 0.005) * length)
            elif relief:
                altitude.append(s.between(-0.02, 0.02) * length)
            else:
                altitude.append(0.0)
        ground = []
        for _ in distance:
            if relief:
                ground.append(0.0 if s.unit() < 0.7 else s.unit() * 0.3)
            else:
                ground.append(s.ground())
        pick = int(s.unit() * 3.0)
        source_gf = 0.0 if pick == 0 else (1.0 if pick == 1 else s.unit())
        terrain = list(zip(distance, altitude))
        tops = []
        for _ in range(int(s.unit() * 4.0)):
            x = s.between(0.0, length)
            k = min(max(sum(1 for d in distance if d <= x), 1), vertices - 1) - 1
            tops.append((x, altitude[k] + s.between(0.5, 25.0)))
        tops.sort(key=lambda t: t[0])
        source = (0.0, altitude[0] + s.between(0.05, 4.0))
        receiver = (length, altitude[-1] + s.between(1.5, 30.0))
        hom, fav = gains(distance, altitude, ground, source, receiver, source_gf, terrain, tops)
        w = worst["relief" if relief else "flat"]
        w[0], w[1] = max(w[0], hom), max(w[1], fav)
    assert worst["flat"][0] <= FLAT_HOMOGENEOUS_GAIN_BOUND_DB, worst
    assert worst["flat"][1] <= FLAT_FAVOURABLE_GAIN_BOUND_DB, worst
    assert worst["relief"][0] <= HOMOGENEOUS_GAIN_BOUND_DB, worst
    assert worst["relief"][1] <= FAVOURABLE_GAIN_BOUND_DB, worst


def test_a_sliver_of_soft_ground_is_hard_ground():
    for state in (HOM, FAV):
        sliver = oracle.ground_attenuation_bands((0.0, 0.0), (0.0, 0.05), (36.5, 4.0), 1e-6, 1e-6, 1e-6, state)
        hard = oracle.ground_attenuation_bands((0.0, 0.0), (0.0, 0.05), (36.5, 4.0), 0.0, 0.0, 0.0, state)
        assert np.all(np.abs(sliver - hard) < 1e-4), (sliver, hard)
