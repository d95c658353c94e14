"""Pins of the FP64 oracle against the reference's own known-answer tests.

The ISO/TR 17534-4 fixture and the Zwicker/atmosphere expectations are read in place from the
reference tree when it is present (they are not copied into this repository); the ray pins restate
the scenarios of physics/src/ray_tests.rs with the constants it asserts.
"""

import json
import math
import re

import numpy as np
import pytest

from conftest import reference_file
from oracle import oracle

BANDS = 8


# ---------------------------------------------------------------------------------------------
# ISO/TR 17534-4 TC01-TC28, direct path, both states, every band within 0.1 dB
# (physics/src/cnossos/iso_tr_17534_4_tests.rs:115-172).

def _parse_case(case, rows, lh, lf):
    """The harness's parse() (iso_tr_17534_4_tests.rs:38-113): cut points as vertices, building
    enter/exit pairs raised as hard roofs, stretch-constant G turned into vertex G."""
    vertices = [(float(p[1]), float(p[2]), float(p[3])) for p in case["cut_points"]]
    terrain = [(v[0], v[1]) for v in vertices]
    walls = case["walls"]
    enter = None
    for wall in walls:
        x, top = float(wall[0]), float(wall[1])
        kind = wall[3]
        if kind == "BUILDING_ENTER":
            enter = (x, top)
        elif kind == "BUILDING_EXIT":
            x0, top0 = enter
            enter = None

            def ground_at(xq, lst):
                previous = lst[0]
                for v in lst:
                    if v[0] >= xq:
                        span = v[0] - previous[0]
                        return previous[1] + (xq - previous[0]) / span * (v[1] - previous[1]) if span > 0 else v[1]
                    previous = v
                return previous[1]

            g_after = [v for v in vertices if v[0] <= x][-1][2]
            z0, z1 = ground_at(x0, vertices), ground_at(x, vertices)
            vertices = [v for v in vertices if not (x0 <= v[0] <= x)]
            vertices += [(x0, z0, 0.0), (x0, top0, 0.0), (x, top, 0.0), (x, z1, g_after)]
            vertices.sort(key=lambda v: v[0])  # stable, as Rust's sort_by
    stepped = []
    for index, (x, z, g) in enumerate(vertices):
        if index > 0:
            stepped.append((x, z, vertices[index - 1][2]))
        stepped.append((x, z, g))
    lh_values = [float(r[lh]) for r in rows]
    lf_values = [float(r[lf]) for r in rows]
    return dict(
        name=case["name"], power=float(case["sound_power_db"]),
        source=(0.0, float(case["source"][2])),
        receiver=(float(case["horizontal_distance_m"]), float(case["receiver"][2])),
        source_gf=float(case["cut_points"][0][3]),
        d=[v[0] for v in stepped], z=[v[1] for v in stepped], g=[v[2] for v in stepped],
        terrain=terrain, tops=[(float(w[0]), float(w[1])) for w in walls], lh=lh_values, lf=lf_values)


def test_iso_tr_17534_4_every_direct_case_within_a_tenth_of_a_decibel():
    path = reference_file("physics/tests/fixtures/cnossos_iso_tr_17534_4_direct.json")
    fixture = json.load(open(path))
    alpha = oracle.alpha_bands(10.0, 70.0)
    columns = fixture["band_columns"]
    lh, lf = columns.index("LH"), columns.index("LF")
    rows = fixture["bands"]
    assert len(rows) == 28 * BANDS
    failures = []
    for raw in fixture["cases"]:
        case_rows = [r for r in rows if r[0] == raw["name"]]
        assert len(case_rows) == BANDS
        case = _parse_case(raw, case_rows, lh, lf)
        direct = math.dist(case["source"], case["receiver"])
        base = [case["power"] - (20 * math.log10(direct) + 11) - alpha[b] * direct / 1000 for b in range(BANDS)]
        att, _ = oracle.state_boundaries(case["d"], case["z"], case["g"], case["source"], case["receiver"],
                                         case["source_gf"], case["terrain"], case["tops"])
        for state, reference in ((0, case["lh"]), (1, case["lf"])):
            for b in range(BANDS):
                level = base[b] - att[state, b]
                if not math.isfinite(level) or abs(level - reference[b]) > 0.1:
                    failures.append(f"{case['name']} state {state} band {b}: {level:.2f} vs {reference[b]:.2f}")
    assert not failures, "\n".join(failures)


def test_ground_split_regression_keeps_every_band_finite():
    """physics/src/cnossos/ground_split_regression_tests.rs:47-77: a source below its side's
    mean plane under two roofs keeps every band finite."""
    value = json.load(open(reference_file("physics/tests/fixtures/cnossos_ground_split_regression.json")))
    att, wog = oracle.state_boundaries(value["distance_m"], value["altitude_m"], value["ground_factor"],
                                       value["source"], value["receiver"], value["source_ground_factor"],
                                       value["terrain_candidates"], value["obstacle_tops"])
    assert np.all(np.isfinite(att)) and np.all(np.isfinite(wog))


# ---------------------------------------------------------------------------------------------
# Air absorption (physics/src/atmosphere.rs:156-183), expectations read from the source.

def _float_list_after(text, anchor):
    start = text.index(anchor)
    block = text[start:text.index("];", start)]
    return [float(v) for v in re.findall(r"-?\d+\.\d+", block.split("[", 1)[1])]


def test_air_absorption_matches_the_iso_tr_and_default_tables():
    text = open(reference_file("physics/src/atmosphere.rs")).read()
    ten = _float_list_after(text, "let expected = [0.12")
    fifteen = _float_list_after(text, "let expected = [0.10")
    np.testing.assert_allclose(oracle.alpha_bands(10.0, 70.0), ten, atol=0.006)
    np.testing.assert_allclose(oracle.alpha_bands(15.0, 70.0), fifteen, atol=0.005)


def test_host_alpha_equals_the_oracle():
    from quietmap_b200.physics import alpha_bands
    np.testing.assert_allclose(alpha_bands(15.0, 70.0), oracle.alpha_bands(15.0, 70.0), rtol=1e-13)


# ---------------------------------------------------------------------------------------------
# Zwicker loudness vs MoSQITo 1.2 (physics/src/loudness.rs:193-265), values read from the source.

def test_zwicker_matches_the_reference_implementation_values():
    text = open(reference_file("physics/src/loudness.rs")).read()
    tests = text[text.index("fn loudness_matches_the_reference_implementation"):]
    quiet = [-60.0] * 28
    one_k = list(quiet)
    one_k[16] = 40.0
    assert abs(oracle.zwicker(one_k) - 0.927) < 0.002
    one_k[16] = 70.0
    assert abs(oracle.zwicker(one_k) - 6.944) < 0.005

    def shifted(octaves, offset):
        thirds = list(quiet)
        for octave, level in enumerate(octaves):
            for third in range(3):
                thirds[4 - 1 + 3 * octave + third] = max(level + offset - 10 * math.log10(3), -60.0)
        return thirds

    road = [float(v) for v in re.search(r"let road = \[([^\]]*)\]", tests).group(1).split(",")]
    for offset, sone in re.findall(r"\((-?\d+\.\d+), (\d+\.\d+)\)", tests[tests.index("for (offset, sone)"):
                                                                         tests.index("let aircraft")]):
        n = oracle.zwicker(shifted(road, float(offset)))
        assert abs(n - float(sone)) / float(sone) < 0.003
    aircraft = [float(v) for v in re.search(r"let aircraft = \[([^\]]*)\]", tests).group(1).split(",")]
    expected = float(re.search(r"\(n - (\d+\.\d+)\)", tests[tests.index("let aircraft"):]).group(1))
    assert abs(oracle.zwicker(shifted(aircraft, -5.0)) - expected) / expected < 0.003
    block = tests[tests.index("let random"):]
    cases = re.findall(r"\[\s*([-\d\.,\s]+?)\s*\],\s*(\d+\.\d+),", block)
    assert len(cases) == 4
    for levels, sone in cases:
        levels = [float(v) for v in levels.split(",") if v.strip()]
        assert len(levels) == 28
        assert abs(oracle.zwicker(levels) - float(sone)) / float(sone) < 0.003


def test_zwicker_silence_is_zero():
    assert oracle.zwicker([-np.inf] * 28) == 0.0


# ---------------------------------------------------------------------------------------------
# Ray pins (physics/src/ray_tests.rs).

def _profile():
    # ray_tests.rs:15-25
    return dict(horizontal_m=100.0, t=[0.0, 0.25, 0.3, 0.5, 0.75, 1.0],
                ground_m=[100.0, 102.0, 105.0, 101.0, 103.0, 100.0],
                ground_factor=[1.0, 0.5, 0.4, 0.0, 0.5, 1.0])


def _ends(**kw):
    # ray_tests.rs:27-36
    ends = dict(source_height_m=4.0, source_ground_m=None, receiver_altitude_m=104.0,
                source_ground_factor=0.5, platform_half_width_m=30.0, own_footprint=1)
    ends.update(kw)
    return ends


def _ray(profile, crossings, ends, p=(0.0, 0.0, 0.0)):
    return oracle.ray_terms(profile["horizontal_m"], profile["t"], profile["ground_m"], profile["ground_factor"],
                            crossings, ends, p, oracle.alpha_bands(15.0, 70.0))


def building(t, h, fp):
    return (t, h, True, True, fp)


def barrier(t, h, fp):
    return (t, h, False, False, fp)


def test_platform_clamps_near_terrain():
    # ray_tests.rs:58-79
    r = _ray(_profile(), [], _ends())
    np.testing.assert_allclose(r["path_d"], [0.0, 25.0, 30.0, 50.0, 75.0, 100.0], atol=1e-9)
    np.testing.assert_allclose(r["path_z"], [100.0, 100.0, 105.0, 101.0, 103.0, 100.0], atol=1e-9)
    np.testing.assert_allclose(r["path_g"], [1.0, 0.5, 0.4, 0.0, 0.5, 1.0], atol=1e-9)


def test_source_on_a_deck():
    # ray_tests.rs:81-105
    r = _ray(_profile(), [], _ends(source_ground_m=150.0))
    np.testing.assert_allclose(r["path_z"], [100.0, 102.0, 105.0, 101.0, 103.0, 100.0], atol=1e-9)
    assert abs(r["slant_m"] - math.hypot(100.0, 50.0)) < 1e-9


def test_own_footprint_skipped_tops_on_interpolated_terrain():
    # ray_tests.rs:107-135
    crossings = [building(0.05, 6.0, 1), building(0.1, 5.0, 3), building(0.12, 5.0, 3), barrier(0.6, 3.0, 2),
                 building(0.9, 6.0, 1), barrier(1.0, 4.0, 4)]
    r = _ray(_profile(), crossings, _ends())
    np.testing.assert_allclose(r["tops"], [(10.0, 105.0), (12.0, 105.0), (60.0, 104.8), (100.0, 104.0)], atol=1e-9)


def test_footprints_containing_a_buildings_source_do_not_screen_it():
    # ray_tests.rs:137-164
    crossings = [building(0.02, 20.0, 5), building(0.05, 20.0, 1), building(0.4, 8.0, 6), building(0.45, 8.0, 6)]
    r = _ray(_profile(), crossings, _ends())
    np.testing.assert_allclose(r["tops"][:, 0], [40.0, 45.0], atol=1e-9)
    r = _ray(_profile(), crossings, _ends(own_footprint=0))
    assert len(r["tops"]) == 4


def test_overlapping_roofs_clip_in_closing_order():
    # ray_tests.rs:166-207
    profile = dict(horizontal_m=100.0, t=[0.0, 0.5, 1.0], ground_m=[100.0] * 3, ground_factor=[1.0, 0.5, 0.0])
    crossings = [building(0.2, 6.0, 11), building(0.4, 6.0, 11), building(0.3, 8.0, 12), building(0.5, 10.0, 12),
                 building(0.25, 7.0, 13), building(0.4, 7.0, 13)]
    r = _ray(profile, crossings, _ends(own_footprint=0))
    np.testing.assert_allclose(r["path_d"], [0.0, 20.0, 20.0, 40.0, 40.0, 40.0, 40.0, 50.0, 50.0, 100.0], atol=1e-9)
    np.testing.assert_allclose(r["path_z"], [100.0, 100.0, 106.0, 106.0, 100.0, 100.0, 109.0, 110.0, 100.0, 100.0],
                               atol=1e-9)
    np.testing.assert_allclose(r["path_g"], [1.0, 0.8, 0.0, 0.0, 0.6, 0.6, 0.0, 0.0, 0.5, 0.0], atol=1e-9)


def _flat(horizontal):
    # ray_tests.rs:209-217
    return dict(horizontal_m=horizontal, t=[k / 10 for k in range(11)], ground_m=[200.0] * 11,
                ground_factor=[0.5] * 11)


def test_flat_ground_transfer_mixes_states_and_absorbs_air():
    # ray_tests.rs:219-273 (dev4 pins to 1e-9)
    ends = dict(source_height_m=1.0, source_ground_m=None, receiver_altitude_m=204.0, source_ground_factor=0.5,
                platform_half_width_m=0.0, own_footprint=0)
    alpha = oracle.alpha_bands(15.0, 70.0)
    hom = _ray(_flat(110.54), [], ends, (0.0, 0.0, 0.0))
    fav = _ray(_flat(110.54), [], ends, (1.0, 1.0, 1.0))
    mixed = _ray(_flat(110.54), [], ends, (0.5, 0.0, 1.0))
    slant = math.hypot(110.54, 3.0)
    assert abs(hom["slant_m"] - slant) < 1e-12
    air = lambda b: 10 ** (-alpha[b] * slant / 1000 / 10)
    assert abs(hom["periods"][0][4] / air(4) - 0.9097167331685742) < 1e-9
    assert abs(fav["periods"][0][4] / air(4) - 1.4125375446227544) < 1e-9
    assert abs(hom["periods"][0][0] / air(0) - 1.4125375446227544) < 1e-9
    for b in range(BANDS):
        expected = 0.5 * hom["periods"][0][b] + 0.5 * fav["periods"][0][b]
        assert abs(mixed["periods"][0][b] - expected) < 1e-12
        assert mixed["periods"][1][b] == hom["periods"][1][b]
        assert mixed["periods"][2][b] == fav["periods"][2][b]


def test_a_wall_between_source_and_receiver_screens():
    # ray_tests.rs:317-349
    profile = _flat(200.0)
    profile["ground_factor"] = [0.0] * 11
    ends = dict(source_height_m=0.05, source_ground_m=None, receiver_altitude_m=204.0, source_ground_factor=0.0,
                platform_half_width_m=0.0, own_footprint=0)
    p = (0.5, 0.5, 0.5)
    open_ = _ray(profile, [], ends, p)
    walled = _ray(profile, [barrier(0.5, 6.0, 9)], ends, p)
    assert 10 * math.log10(open_["periods"][0][4] / walled["periods"][0][4]) > 10.0


def test_crests_thin_to_the_highest_of_each_150_m():
    # ray_tests.rs:351-389
    length = 1000.0
    terrain = [(10.0 * k, 5.0 if k % 8 == 3 else 0.0) for k in range(101)]
    crests = [tuple(p) for p in oracle.crests_of(terrain, length)]
    middle = lambda x: 300.0 < x < length - 300.0
    assert all(p in crests for p in terrain if not middle(p[0]))
    assert [p for p in crests if middle(p[0])] == [(350.0, 5.0), (510.0, 5.0), (670.0, 5.0)]
    shifted = list(terrain)
    shifted[30] = (300.0001, shifted[30][1])
    fewer = terrain[:1] + terrain[2:]
    beyond = lambda lst: [tuple(p) for p in lst if p[0] >= 320.0]
    for other in (shifted, fewer):
        assert beyond(oracle.crests_of(other, length)) == beyond(crests)


# ---------------------------------------------------------------------------------------------
# Level-distribution bins (popup/src/distribution.rs:69-72).

def test_level_bins_round_and_clamp_into_the_grid():
    assert oracle.level_bin(-30.0, -30.0, 0.1, 1800) == 0
    assert oracle.level_bin(-100.0, -30.0, 0.1, 1800) == 0
    assert oracle.level_bin(float("nan"), -30.0, 0.1, 1800) == 0
    assert oracle.level_bin(500.0, -30.0, 0.1, 1800) == 1799
    assert oracle.level_bin(-29.95, -30.0, 0.1, 1800) == round((-29.95 + 30.0) / 0.1)
    assert oracle.level_bin(60.04, -30.0, 0.1, 1800) == 900
    counts = oracle.level_histogram(np.array([-40.0, 0.0, 0.0, 200.0]), -30.0, 0.1, 1800)
    assert counts.sum() == 4 and counts[0] == 1 and counts[300] == 2 and counts[1799] == 1


def test_lden_of_60_55_50_is_60():
    # physics/src/bands.rs:79-83
    from quietmap_b200.physics import lden_weights
    e = lden_weights() @ (10.0 ** (np.array([60.0, 55.0, 50.0]) / 10))
    assert abs(10 * math.log10(e) - 60.0) < 0.01
