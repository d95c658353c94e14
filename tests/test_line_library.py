"""The library's line quadrature and receiver skyline (qm_line.cuh, qm_skyline.cuh: one source
for the host and the device), run on the host through the C ABI and checked against the oracle
to the bit: random pieces near and far with random obstacle arcs in front of them; the skyline
index against the oracle's scene skyline (itself pinned to the reference's skyline tests);
wide buckets querying the index; and the entry points' errors and capacity limits."""

import math

import numpy as np
import pytest

from helpers import Stock, square
from oracle import oracle
from quietmap_b200 import abi, native


def _random_piece(rng):
    """A piece within 5-300 m of the receiver, some seen under a wide angle, some tilted."""
    centre = rng.uniform(-300.0, 300.0, 2)
    if rng.random() < 0.5:
        centre *= rng.uniform(0.01, 0.1)
    direction = rng.uniform(-math.pi, math.pi)
    half = rng.uniform(0.0005, 200.0) if rng.random() < 0.9 else rng.uniform(0.0, 0.001)
    z = rng.uniform(-8.0, 2.0, 2)
    start = [centre[0] - half * math.cos(direction), centre[1] - half * math.sin(direction), z[0]]
    end = [centre[0] + half * math.cos(direction), centre[1] + half * math.sin(direction), z[1]]
    return start, end


def _random_arcs(rng, n):
    lo = rng.uniform(-math.pi, math.pi, n)
    width = rng.uniform(0.0, 0.6, n)
    nearest = rng.uniform(0.3, 150.0, n)
    return np.stack([lo, lo + width, nearest], axis=1)


def test_nodes_match_the_oracle_to_the_bit():
    rng = np.random.default_rng(2024)
    placed = 0
    for _ in range(3000):
        start, end = _random_piece(rng)
        arcs = _random_arcs(rng, int(rng.integers(0, 12)))
        want = oracle.line_nodes(start, end, arcs)
        nodes, figures = native.line_quadrature_nodes(start, end, arcs=arcs)
        if want is None:
            assert len(nodes) == 0 and figures["length_m"] < 1e-3
            continue
        along, weight, on_ray = want
        assert np.array_equal(nodes["along_m"], along)
        assert np.array_equal(nodes["weight_rad"], weight)
        assert np.array_equal(nodes["obstacles_on_ray"].astype(bool), on_ray)
        g = oracle.line_geometry(start, end)
        assert figures["subtended_angle_rad"] == g["subtended_rad"]
        assert figures["divergence_factor"] == g["divergence_factor"]
        placed += len(along) > 5
    assert placed > 100, "wide buckets with obstacles in front place their own nodes"


def _scene(seed):
    rng = np.random.default_rng(seed)
    stock = Stock()
    for fp in range(1, 51):
        cx, cy = rng.uniform(-150.0, 150.0, 2)
        if rng.random() < 0.7:
            stock.building(fp, float(rng.uniform(1.0, 25.0)), [square(cx, cy, rng.uniform(2.0, 15.0))])
        else:
            points = [(cx, cy)] + [tuple(rng.uniform(-150.0, 150.0, 2)) for _ in range(int(rng.integers(1, 4)))]
            stock.wall(fp, float(rng.uniform(0.02, 6.0)), points)
    return stock


def test_the_skyline_index_hands_over_the_oracles_arcs():
    """Same arcs in the same order, bit for bit, over receivers, wedges (some past pi), radii and
    sight-line floors; an unbounded radius walks only the rows the index holds."""
    stock = _scene(17)
    scene = stock.scene()
    ora = oracle.OracleScene(scene)
    sky = native.Skyline.of_scene(scene)
    cells, runs = sky.counts()
    assert cells > 100 and runs >= cells
    rng = np.random.default_rng(9)
    total = 0
    for _ in range(120):
        r = stock.steps(rng.uniform(-160.0, 160.0, 2))
        lo = rng.uniform(-math.pi, math.pi)
        hi = lo + rng.uniform(0.001, 3.1)
        radius, floor = rng.uniform(1.0, 300.0), float(rng.choice([0.0, 0.05, 2.0, 12.0, 30.0]))
        got = sky.arcs(r, lo, hi, radius, floor)
        want = ora.skyline_arcs(r, lo, hi, radius, floor)
        assert np.array_equal(got, want), (r, lo, hi, radius, floor)
        total += len(got)
    assert total > 1000
    r = stock.steps((0.0, 0.0))
    assert np.array_equal(sky.arcs(r, 0.2, 2.9, 1e300, 0.0), ora.skyline_arcs(r, 0.2, 2.9, 2000.0, 0.0))
    assert len(sky.arcs(r, 0.2, 2.9, 0.0, 0.0)) == 0
    sky.close()


def test_wide_buckets_query_the_index_as_the_line_evaluation_does():
    """Nodes over the index from a receiver, with the sight line's floor (the source's height in
    the line evaluation, popup/src/evaluate.rs:225-242), equal the oracle's nodes over its own
    scene skyline to the bit, bucket by bucket."""
    stock = _scene(23)
    scene = stock.scene()
    ora = oracle.OracleScene(scene)
    sky = native.Skyline.of_scene(scene)
    rng = np.random.default_rng(4)
    placed = 0
    for _ in range(300):
        r = stock.steps(rng.uniform(-120.0, 120.0, 2))
        start, end = _random_piece(rng)
        floor = float(rng.choice([0.05, 0.5, 4.0]))
        want = ora.line_nodes(r, start, end, floor)
        nodes, _ = native.line_quadrature_nodes(start, end, skyline=sky, receiver_xy=r, floor_m=floor)
        if want is None:
            assert len(nodes) == 0
            continue
        assert np.array_equal(nodes["along_m"], want[0]) and np.array_equal(nodes["weight_rad"], want[1])
        assert np.array_equal(nodes["obstacles_on_ray"].astype(bool), want[2])
        placed += len(nodes) > 5
    assert placed > 20
    sky.close()


def test_errors_and_limits():
    start, end = [-125.0, 20.0, 0.0], [125.0, 20.0, 0.0]
    with pytest.raises(native.QmError) as err:
        native.line_quadrature_nodes(start, end, cap=2)
    assert err.value.status == abi.QM_ERR_CAPACITY and "5 nodes" in str(err.value)
    with pytest.raises(native.QmError) as err:
        native.line_quadrature_nodes([0.0, math.nan, 0.0], end)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    nodes, figures = native.line_quadrature_nodes([1.0, 2.0, 3.0], [1.0, 2.0, 3.0])
    assert len(nodes) == 0 and figures["length_m"] == 0.0

    # The most nodes one piece takes stays within the stated bound: a dense comb of thin arcs.
    comb = [(math.radians(20.0 + 0.7 * k), math.radians(20.0 + 0.7 * k + 0.2), 5.0) for k in range(200)]
    nodes, _ = native.line_quadrature_nodes([-1000.0, 20.0, 0.0], [1000.0, 20.0, 0.0], arcs=comb)
    assert 5 < len(nodes) <= abi.LINE_MAX_NODES

    vertices = np.array([[0, 0], [100, 0], [100, 100]], np.int32)
    outlines = np.zeros(1, dtype=abi.OUTLINE_DTYPE)
    outlines[0] = (1, 3, 7, 5.0, 0)
    with pytest.raises(native.QmError) as err:
        native.Skyline(vertices, outlines, 0.1)
    assert err.value.status == abi.QM_ERR_ARGUMENT and "outline 0" in str(err.value)
    outlines[0] = (0, 3, 7, 5.0, 0)
    with pytest.raises(native.QmError) as err:
        native.Skyline(vertices, outlines, 0.0)
    assert err.value.status == abi.QM_ERR_ARGUMENT
    sky = native.Skyline(vertices, outlines, 0.1)
    assert sky.counts() == (2, 2), "(100, 100) north is row -1 of the south-growing frame"
    # From the east, an edge through two cells is handed over once per cell.
    arcs = sky.arcs((300, 50), 2.0, 4.0, 500.0, 0.0)
    assert len(arcs) == 3 and np.array_equal(arcs[0], arcs[2])
    with pytest.raises(native.QmError) as err:
        sky.arcs((300, 50), 2.0, 4.0, 500.0, 0.0, cap=1)
    assert err.value.status == abi.QM_ERR_CAPACITY and "3 arcs" in str(err.value)
    empty = native.Skyline(np.zeros((0, 2), np.int32), np.zeros(0, dtype=abi.OUTLINE_DTYPE), 0.1)
    assert empty.counts() == (0, 0) and len(empty.arcs((0, 0), 0.0, 1.0, 1e9, 0.0)) == 0
