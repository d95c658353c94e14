"""The oracle's state rays and rubber band (physics/src/cnossos/rubber_band.rs), pinned to the
reference's own tests (physics/src/cnossos/rubber_band_tests.rs): path differences against the
printed formulas on 20,000 seeded geometries, the arcs of the downwind band, the band as the
upper envelope of the state's rays, and equal-distance crossings."""

import math

from oracle import oracle

HOM, FAV = 0, 1


def _unit_stream(seed):
    """The tests' xorshift generator: uniform [0, 1) from the top 53 bits."""
    mask = (1 << 64) - 1
    while True:
        seed ^= (seed << 13) & mask
        seed ^= seed >> 7
        seed ^= (seed << 17) & mask
        yield (seed >> 11) / float(1 << 53)


def chord_altitude(a, b, x):
    return a[1] + (b[1] - a[1]) * (x - a[0]) / (b[0] - a[0])


def printed(state, radius, start, points, end):
    """(2.5.26) and (2.5.27) as printed: arcs by asin, lengths summed directly
    (rubber_band_tests.rs:7-39)."""
    def arc(a, b):
        chord = math.hypot(b[0] - a[0], b[1] - a[1])
        return chord if state == HOM else 2.0 * radius * math.asin(min(chord / (2.0 * radius), 1.0))
    along = arc(start, points[0]) + arc(points[-1], end)
    for p, q in zip(points[:-1], points[1:]):
        along += arc(p, q)
    excess = along - arc(start, end)
    if len(points) > 1:
        return excess
    first = points[0]
    chord = chord_altitude(start, end, first[0])
    if first[1] >= chord:
        return excess
    if state == HOM:
        return -excess
    a = (first[0], chord)
    return 2.0 * arc(start, a) + 2.0 * arc(a, end) - arc(start, first) - arc(first, end) - arc(start, end)


def test_path_differences_match_the_printed_formulas_for_images_beyond_the_ends():
    unit = _unit_stream(0x9E37_79B9_7F4A_7C15)
    u = lambda: next(unit)
    for case in range(20_000):
        length = 5.0 + 3_000.0 * u()
        source = (0.0, 50.0 * u())
        receiver = (length, 50.0 * u())
        shift = (u() - 0.5) * 0.8 * length
        depth = -20.0 * u()
        start = (shift, depth) if case % 3 == 0 else source
        end = (length + shift, depth) if case % 3 == 1 else receiver
        if end[0] - start[0] < 1.0:
            continue
        count = 1 + case % 3
        points = []
        for k in range(count):
            x = length * (k + u()) / count
            points.append((x, chord_altitude(start, end, x) + (u() - 0.4) * 10.0))
        for state in (HOM, FAV):
            ray = oracle.StateRay(state, source, receiver)
            radius = max(1000.0, 8.0 * math.hypot(receiver[0] - source[0], receiver[1] - source[1]))
            got, want = ray.path_difference(start, points, end), printed(state, radius, start, points, end)
            assert abs(got - want) < 1e-7 * (1.0 + abs(want)), (case, state, got, want)


def test_the_downwind_band_is_made_of_arcs():
    ray = oracle.StateRay(FAV, (0.0, 0.0), (1_000.0, 0.0), radius_m=8_000.0)
    blocked, points, _ = ray.diffraction_path([(250.0, 100.0), (600.0, 62.2)])
    assert blocked and points == [(250.0, 100.0)]
    _, points, _ = ray.diffraction_path([(250.0, 100.0), (600.0, 62.5)])
    assert points == [(250.0, 100.0), (600.0, 62.5)]


def test_the_band_is_the_upper_envelope_of_the_states_rays():
    unit = _unit_stream(0x2545_F491_4F6C_DD1D)
    u = lambda: next(unit)
    for case in range(3_000):
        length = 50.0 + 4_000.0 * u()
        source = (0.0, 30.0 * u())
        receiver = (length, 30.0 * u())
        candidates = []
        for _ in range(1 + case % 12):
            x = length * (0.01 + 0.98 * u())
            z = 60.0 * u()
            z += 0.02 * length * u()
            candidates.append((x, z))
        candidates.sort(key=lambda p: p[0])
        for state in (HOM, FAV):
            ray = oracle.StateRay(state, source, receiver)
            blocked, points, blocking = ray.diffraction_path(candidates)
            if not blocked:
                continue
            under = lambda a, b, p: p[1] <= ray.altitude(a, b, p[0]) + 1e-9
            band = [source] + points + [receiver]
            for a, p, b in zip(band[:-2], band[1:-1], band[2:]):
                assert not under(a, b, p), (case, state)
            for x, z in blocking:
                if (x, z) in band:
                    continue
                nxt = next(i for i, p in enumerate(band) if p[0] > x)
                assert under(band[nxt - 1], band[nxt], (x, z)), (case, state)


def test_equal_distance_crossings_keep_only_the_highest():
    source, receiver = (0.0, 0.0), (100.0, 0.0)
    for state in (HOM, FAV):
        ray = oracle.StateRay(state, source, receiver)
        blocked, points, _ = ray.diffraction_path([(50.0, 20.0), (50.0, 15.0), (50.0, 25.0)])
        assert blocked and points == [(50.0, 25.0)], state
    low_first = [(90.0, 100.0), (90.5, 99.0), (91.0, 10.0), (91.0, 60.0)]
    high_first = [(90.0, 100.0), (90.5, 99.0), (91.0, 60.0), (91.0, 10.0)]
    for state in (HOM, FAV):
        ray = oracle.StateRay(state, source, receiver)
        _, from_low, _ = ray.diffraction_path(low_first)
        blocked, from_high, _ = ray.diffraction_path(high_first)
        assert blocked and from_low == from_high, state
        if state == FAV:
            assert from_low == [(90.0, 100.0), (90.5, 99.0)]
