"""The line-piece quadrature (physics/src/line.rs), pinned to the reference's own tests
(physics/src/line_tests.rs): free-field exactness against a numeric point sum, the
normalisation, the in-plane angle, the perpendicular floor, and the bucket and wide-bucket nodes.
Every test runs twice: on the oracle's restatement and on the library's shared host/device
quadrature through its C ABI (qm_line_quadrature_nodes, run on the host; no GPU)."""

import math
import types

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import native


def _library_nodes(start, end, arcs=()):
    nodes, _ = native.line_quadrature_nodes(start, end, arcs=arcs)
    if len(nodes) == 0:
        return None
    return nodes["along_m"], nodes["weight_rad"], nodes["obstacles_on_ray"].astype(bool)


def _library_geometry(start, end):
    nodes, figures = native.line_quadrature_nodes(start, end)
    if len(nodes) == 0:
        return None
    return dict(length_m=figures["length_m"], subtended_rad=figures["subtended_angle_rad"],
                divergence_factor=figures["divergence_factor"])


IMPLEMENTATIONS = {
    "oracle": types.SimpleNamespace(line_nodes=oracle.line_nodes, line_geometry=oracle.line_geometry),
    "library": types.SimpleNamespace(line_nodes=_library_nodes, line_geometry=_library_geometry),
}
IMPL = IMPLEMENTATIONS["oracle"]


@pytest.fixture(autouse=True, params=sorted(IMPLEMENTATIONS))
def implementation(request):
    global IMPL
    IMPL = IMPLEMENTATIONS[request.param]
    yield request.param
    IMPL = IMPLEMENTATIONS["oracle"]

DIVERGENCE = 12.589254117941673  # 10^1.1
BUCKETS = 5
ONE_BUCKET_SPAN = 3.0 * math.pi / 180.0


def db(ratio):
    return 10.0 * math.log10(ratio)


def relative(point, receiver):
    return [point[k] - receiver[k] for k in range(3)]


def free_field_energy(start, end, receiver):
    """sum(dphi) / (10^1.1 d_perp) per unit L_W' (line_tests.rs:20-27)."""
    s, e = relative(start, receiver), relative(end, receiver)
    _, weight, _ = IMPL.line_nodes(s, e)
    return weight.sum() * IMPL.line_geometry(s, e)["divergence_factor"]


def point_sum_energy(start, end, receiver, steps=400_000):
    """The incoherent point sum, 20 lg r + 11 per point, by a fine midpoint rule per horizontal
    metre (line_tests.rs:29-46)."""
    start, end, receiver = (np.asarray(v, dtype=np.float64) for v in (start, end, receiver))
    along = end - start
    f = (np.arange(steps) + 0.5) / steps
    p = start[None, :] + f[:, None] * along[None, :] - receiver[None, :]
    return (1.0 / (p * p).sum(axis=1)).sum() * math.hypot(along[0], along[1]) / steps / DIVERGENCE


def test_free_field_quadrature_is_the_exact_point_sum_on_any_geometry():
    scenes = [([-125.0, 0.0, 0.05], [125.0, 0.0, 0.05], [0.0, 50.0, 4.0]),
              ([0.0, 0.0, 0.05], [250.0, 0.0, 0.05], [500.0, 30.0, 4.0]),
              ([-125.0, 0.0, 0.05], [125.0, 0.0, 0.05], [0.0, 1.0, 4.0]),
              ([0.0, 0.0, 0.5], [250.0, 0.0, 12.0], [40.0, 90.0, 4.0]),
              ([2000.0, 0.0, 0.05], [2250.0, 0.0, 0.05], [0.0, 45.0, 4.0]),
              ([-5.0, 0.0, 0.05], [5.0, 0.0, 0.05], [0.0, 1.0, 4.0])]
    for start, end, receiver in scenes:
        got, exact = free_field_energy(start, end, receiver), point_sum_energy(start, end, receiver)
        assert abs(db(got / exact)) < 1e-6, (start, end, receiver, db(got / exact))


def test_the_line_is_1_9533_db_above_the_retired_two_pi_chain():
    theta = 2.0 * math.atan(125.0 / 1000.0)
    retired = -db(2.0 * math.pi * 1000.0) + db(theta / math.pi)
    gap = db(free_field_energy([-125.0, 0.0, 4.0], [125.0, 0.0, 4.0], [0.0, 1000.0, 4.0])) - retired
    assert abs(gap - 1.9533) < 0.0005, gap
    infinite = db(free_field_energy([-1e7, 0.0, 4.0], [1e7, 0.0, 4.0], [0.0, 100.0, 4.0]))
    assert abs(infinite + db(100.0) + 6.0285) < 1e-3, infinite


def test_the_in_plane_angle_replaces_the_horizontal_one_beside_a_short_elevated_line():
    slant = math.sqrt(1.0 + 3.95 * 3.95)
    retired = -db(2.0 * math.pi * slant) + db(2.0 * math.atan(5.0) / math.pi)
    normalization = db(2.0 * math.pi * math.pi / DIVERGENCE)
    excess = retired + normalization - db(free_field_energy([-5.0, 0.0, 0.05], [5.0, 0.0, 0.05], [0.0, 1.0, 4.0]))
    assert abs(excess - 1.899) < 0.002, excess


def test_a_receiver_on_the_line_reads_it_half_a_metre_away():
    g = IMPL.line_geometry([-125.0, 0.0, 0.0], [125.0, 0.0, 0.0])
    assert g["divergence_factor"] == 1.0 / (DIVERGENCE * 0.5)
    assert IMPL.line_geometry([1.0, 2.0, 3.0], [1.0, 2.0, 3.0]) is None


def test_nodes_are_uniform_in_the_in_plane_angle():
    s, e = [-125.0, 20.0, -3.95], [125.0, 20.0, -3.95]
    along, _, _ = IMPL.line_nodes(s, e)
    assert len(along) == BUCKETS
    angles = [oracle.line_in_plane_angle_at(s, e, a) for a in along]
    step = IMPL.line_geometry(s, e)["subtended_rad"] / BUCKETS
    for a, b in zip(angles[:-1], angles[1:]):
        assert abs(b - a - step) < 1e-12
    assert abs(along[2] - 125.0) < 1e-9, "the middle node faces the receiver"


def test_a_piece_seen_under_a_small_angle_takes_one_node():
    s, e = [-10.0, 1000.0, -3.95], [10.0, 1000.0, -3.95]
    g = IMPL.line_geometry(s, e)
    assert g["subtended_rad"] < ONE_BUCKET_SPAN
    along, weight, _ = IMPL.line_nodes(s, e)
    assert len(along) == 1
    assert abs(weight[0] - g["subtended_rad"]) < 1e-15
    assert abs(along[0] - 10.0) < 1e-9


def test_a_wall_in_front_of_a_wide_bucket_places_blocked_and_clear_nodes():
    s, e = [-125.0, 20.0, 0.0], [125.0, 20.0, 0.0]
    g = IMPL.line_geometry(s, e)
    for nearest in (10.0, 0.5):
        wall = (math.radians(80.0), math.radians(100.0), nearest)
        along, weight, on_ray = IMPL.line_nodes(s, e, [wall])
        assert len(along) > BUCKETS
        assert abs(weight.sum() - g["subtended_rad"]) < 1e-12
        azimuth = np.degrees(np.arctan2(np.full_like(along, 20.0), s[0] + along))
        clear = ~on_ray
        assert clear.any(), "the gaps beside the wall are clear nodes"
        assert not np.any((azimuth[clear] >= 80.0) & (azimuth[clear] <= 100.0))
        assert np.any(on_ray & (azimuth >= 80.0) & (azimuth <= 100.0))
