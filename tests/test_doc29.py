"""The Doc 29 oracle pinned to the reference's known answers (physics/src/doc29/corrections_tests.rs,
npd_tests.rs) and checked on the seeded flight workload's own NPD tables."""

import math

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import scenes

FT = 0.3048


def test_speed_correction_zero_at_reference_and_3db_at_half_speed():
    # corrections_tests.rs:9-13
    assert abs(oracle.speed_correction_db(160.0, 160.0)) < 1e-12
    assert abs(oracle.speed_correction_db(160.0, 80.0) - 3.0103) < 1e-4
    assert oracle.speed_correction_db(160.0, 5.0) == 0.0


def test_finite_segment_alongside_behind_and_infinite():
    # corrections_tests.rs:16-27
    alongside = oracle.finite_segment_energy_fraction(500.0, 1000.0, 370.0)
    assert 0.1 < alongside < 1.0
    assert oracle.finite_segment_energy_fraction(-500.0, 1000.0, 370.0) < 10.0 ** -0.5
    assert abs(oracle.finite_segment_energy_fraction(500_000.0, 1_000_000.0, 370.0) - 1.0) < 1e-3
    assert abs(oracle.finite_segment_energy_fraction(0.0, 1_000_000.0, 370.0) - 0.5) < 1e-3


@pytest.mark.parametrize("height,lateral,expected", [(100.0, 1000.0, 5.326), (100.0, 8000.0, 9.901),
                                                     (-50.0, 200.0, 4.988)])
def test_lateral_attenuation_matches_doc29(height, lateral, expected):
    # corrections_tests.rs:38-50 (Doc 29 Eq. 4-17/4-18)
    assert abs(oracle.lateral_attenuation_db(height, lateral) - expected) < 0.001


def test_lateral_attenuation_overhead_grazing_and_sign():
    # corrections_tests.rs:30-35, 52-62
    assert oracle.lateral_attenuation_db(1000.0, 0.0) == 0.0
    assert 10.0 < oracle.lateral_attenuation_db(1.0, 2000.0) < 10.9
    for lateral in (0.0, 5.0, 100.0, 913.0, 915.0, 16000.0):
        for height in (-3000.0, -1.0, 0.0, 1.0, 50.0, 800.0, 12000.0):
            assert oracle.lateral_attenuation_db(height, lateral) >= 0.0


def test_installation_peaks_below_its_bound():
    # corrections_tests.rs:64-93; the bound is corrections.rs:13 (0.4014 dB)
    wing_peak = 0.0
    for tenth in range(901):
        angle = math.radians(tenth / 10.0)
        h, s = 1000.0 * math.sin(angle), 1000.0
        wing_peak = max(wing_peak, oracle.installation_energy_gain(0, h, s))
        assert oracle.installation_energy_gain(1, h, s) <= 1.0 + 1e-12
        assert oracle.installation_energy_gain(2, h, s) == 1.0
    assert 0.40 < 10.0 * math.log10(wing_peak) < 0.4014
    below = oracle.installation_energy_gain(0, -300.0, 1000.0)
    assert abs(10.0 * math.log10(below) - 10.0 * 0.062 * math.log10(0.0039)) < 1e-12


def _curves():
    f = scenes.flights_square(n_flights=4, receivers=8)
    for t in f.types:
        for op in range(2):
            for r in range(10):
                yield np.asarray(t["sel_db"][op, r], np.float64)


def test_npd_reads_table_values_and_interpolates_between():
    # npd_tests.rs:19-34
    for curve in _curves():
        alpha = oracle.tail_absorption(curve)
        for k, d in enumerate(scenes.NPD_DISTANCES_FT):
            assert abs(oracle.npd_level(curve, d * FT, alpha) - curve[k]) < 1e-9
        mid = oracle.npd_level(curve, 1500.0 * FT, 0.0)
        assert curve[4] <= mid <= curve[3]


def test_npd_extrapolates_to_100_ft_and_clamps_below():
    # npd_tests.rs:36-45: the first interval extended down to 100 ft is 2 c0 - c1
    for curve in _curves():
        at100 = oracle.npd_level(curve, 100.0 * FT, 0.0)
        assert abs(at100 - (2.0 * curve[0] - curve[1])) < 1e-9
        assert oracle.npd_level(curve, 5.0, 0.0) == at100


def test_npd_tail_is_continuous_and_its_absorption_small():
    # npd_tests.rs:54-80
    last = 25000.0 * FT
    for curve in _curves():
        alpha = oracle.tail_absorption(curve)
        assert 0.0 <= alpha <= 0.003 + 0.0025  # seeded tables carry 0.005 dB/m of their own slope
        for s in (last * (1 - 1e-9), last * (1 + 1e-9)):
            assert abs(oracle.npd_level(curve, s, alpha) - curve[9]) < 1e-6
        # beyond the table the level keeps falling with spreading and absorption
        assert oracle.npd_level(curve, 2 * last, alpha) < curve[9] - 6.0


def _one_segment_scene(z=300.0, power=5.0, length=1000.0, speed=80.0, installation=2):
    from quietmap_b200 import abi
    f = scenes.flights_square(n_flights=1, segments_per_flight=1, n_types=1, receivers=8, spacing_m=100.0)
    f.types["installation"] = installation
    s = f.segments
    s["start"] = (-length / 2, 0.0, z)
    s["end"] = (length / 2, 0.0, z)
    s["power"], s["speed_mps"], s["departure"], s["flight"], s["type"] = power, speed, 1, 0, 0
    f.grid = dict(origin_m=(0.0, 0.0), spacing_m=100.0, nx=8, ny=1, receiver_height_m=0.0, reach_m=0.0,
                  duration_s=1.0)
    return f


def test_flight_grid_overhead_reads_the_npd_with_speed_and_finite_corrections():
    # A receiver right under the middle of a level segment: slant = altitude, no lateral attenuation,
    # propeller installation (no gain), Delta_F of a segment seen from its middle.
    f = _one_segment_scene()
    lae, thirds, sone = oracle.flight_grid(f)
    t = f.types[0]
    row_lo, row_hi = np.asarray(t["sel_db"][1, 5], np.float64), np.asarray(t["sel_db"][1, 6], np.float64)
    sel = oracle.npd_level(row_lo, 300.0, oracle.tail_absorption(row_lo))
    v_ref = float(t["v_ref_kt"])
    dur = np.asarray(t["sel_db"][1, 5], np.float64) - np.asarray(t["lamax_db"][1, 5], np.float64)
    from quietmap_b200.scenes import NPD_DISTANCES_FT
    # scaled distance: d0 * 10^(interp(SEL - LAmax)/10), d0 = 2/pi * V_ref * 1 s
    logd = np.log10(NPD_DISTANCES_FT * FT)
    dl = 2.0 / math.pi * v_ref * 1852.0 / 3600.0 * 10.0 ** (np.interp(math.log10(300.0), logd, dur) / 10.0)
    expected = (sel + oracle.speed_correction_db(v_ref, 80.0 * 3600.0 / 1852.0)
                + 10.0 * math.log10(oracle.finite_segment_energy_fraction(500.0, 1000.0, dl)))
    assert abs(lae[0] - expected) < 1e-6
    assert lae[1] < lae[0] and np.all(np.diff(lae) < 0)
    assert sone[0] > sone[-1] > 0.0


def test_flight_grid_reach_culls_whole_flights():
    f = _one_segment_scene()
    f.grid["reach_m"] = 250.0
    lae, _, _ = oracle.flight_grid(f)
    # cells at x <= 750 m are within 250 m of the flight's box [-500, 500]
    assert np.all(np.isfinite(lae[:8][np.arange(8) * 100.0 <= 750.0]))
    assert np.all(np.isneginf(lae[np.arange(8) * 100.0 > 750.0]))


def test_flight_grid_thirds_carry_the_lae_through_the_a_weighting():
    f = scenes.flights_square(n_flights=20, receivers=16, spacing_m=500.0)
    lae, thirds, sone = oracle.flight_grid(f)
    aw = np.array([-44.7, -39.4, -34.6, -30.2, -26.2, -22.5, -19.1, -16.1, -13.4, -10.9, -8.6, -6.6, -4.8, -3.2,
                   -1.9, -0.8, 0.0, 0.6, 1.0, 1.2, 1.3, 1.2, 1.0, 0.5, -0.1, -1.1, -2.5, -4.3])
    la = 10.0 * np.log10(np.sum(10.0 ** ((thirds + aw) / 10.0), axis=1))
    np.testing.assert_allclose(la, lae - 10.0 * math.log10(f.grid["duration_s"]), atol=1e-9)
    np.testing.assert_allclose(sone, oracle.zwicker_many(thirds), rtol=1e-12)
