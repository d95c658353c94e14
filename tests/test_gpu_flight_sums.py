"""Batch::flight_sums on the device (qm_flight_boxes_upload, qm_flight_sums) against the FP64 oracle
(oracle/qm_oracle_doc29.cpp: FlightBoxes::sums per request, tile_flight_passes over each segment's
boxes, box_sel_at_receiver through the point's horizons).

The boxes are the flight workload's flights summed into fine and far cells; the points stand on the
square with synthetic terrain and building horizons. Every request band's energy per period and its
pass classes' energies and passing shares agree within 1e-8 relative, and each pass lands in the
oracle's class. The bound is the reference's own rounding: its finite-segment fraction subtracts two
arctangent terms near pi/2 for a far piece, so one unit in the last place of either arctangent
(the device's or the C library's) moves a far box's energy by up to a few 1e-9."""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu

RTOL = 1e-8


@pytest.fixture(scope="module")
def world():
    return scenes.flight_boxes_square(seed=9, n_flights=300, receivers=256)


def _compare(got, want, label):
    classes = slice(abi.PERIODS, abi.PERIODS + abi.PERIODS * abi.PASS_CLASSES)
    assert np.array_equal(got[:, classes] != 0.0, want[:, classes] != 0.0), label
    scale = np.maximum(np.abs(want), 1e-300)
    err = np.abs(got - want) / scale
    err[want == 0.0] = np.abs(got[want == 0.0])
    assert err.max() < RTOL, (label, float(err.max()), np.unravel_index(err.argmax(), err.shape))
    return float(err.max())


@pytest.mark.parametrize("lattice", ["exact", "hum", "near"])
def test_flight_sums_match_the_oracle(world, lattice):
    rng = np.random.default_rng(23)
    xy = rng.uniform(500.0, world.side_m - 500.0, (40, 2))
    if lattice == "exact":
        req = dict(weights=(abi.FLIGHT_WEIGHT_ONE, None))
    elif lattice == "hum":
        req = dict(weights=(abi.FLIGHT_WEIGHT_FAR, abi.FLIGHT_WEIGHT_ONE), coarse_m=400.0)
    else:
        req = dict(weights=(abi.FLIGHT_WEIGHT_NEAR, None), coarse_m=900.0, within_m=2700.0)
    points, hz, segs, n_sums = scenes.flight_requests(world, xy, impedance_gain=0.97, seed=29, **req)
    points["altitude_m"] = rng.uniform(0.0, 300.0, len(points))
    ctx = native.Context(0)
    dev = ctx.flight_boxes(world.boxes)
    got, st = dev.sums(points, hz, segs, n_sums, stats=True)
    want, heard = oracle.flight_sums(world.boxes, points, hz, segs, n_sums)
    assert st["boxes_heard"] == heard and st["box_reads"] == int(segs["count"].sum())
    worst = _compare(got, want, lattice)
    print(f"{lattice}: {len(segs)} segments, {st['box_reads']} box reads, {heard} heard, "
          f"max relative error {worst:.2e}, {st['kernel_ms']:.2f} ms")
    dev.close()
    ctx.close()


def test_free_field_helicopters_and_unnamed_bands(world):
    rng = np.random.default_rng(31)
    xy = rng.uniform(0.0, world.side_m, (12, 2))
    points, _, segs, n_sums = scenes.flight_requests(world, xy, horizons=False, impedance_gain=1.3)
    boxes = world.boxes.copy()
    boxes["helicopter"] = np.arange(len(boxes)) % 2
    ctx = native.Context(0)
    dev = ctx.flight_boxes(boxes)
    got = dev.sums(points, None, segs, n_sums + 3)
    want, _ = oracle.flight_sums(boxes, points, None, segs, n_sums + 3)
    _compare(got, want, "free field")
    assert not got[n_sums:].any() and not got[1::2].any()
    # No segments: every band reads zero.
    assert not dev.sums(points, None, segs[:0], 5).any()
    dev.close()
    ctx.close()


def test_shared_points_and_interleaved_sums(world):
    """Segments of one sum naming several points, and sums in no order: the device reads each
    segment's own point and horizons."""
    rng = np.random.default_rng(37)
    xy = rng.uniform(1000.0, world.side_m - 1000.0, (6, 2))
    points, hz, segs, _ = scenes.flight_requests(world, xy)
    segs = segs.copy()
    segs["sum"] = rng.integers(0, 4, len(segs))
    order = rng.permutation(len(segs))
    segs = segs[order]
    ctx = native.Context(0)
    dev = ctx.flight_boxes(world.boxes)
    got = dev.sums(points, hz, segs, 4)
    want, _ = oracle.flight_sums(world.boxes, points, hz, segs, 4)
    _compare(got, want, "interleaved")
    dev.close()
    ctx.close()


def test_bad_arguments_fail_loudly(world):
    points, hz, segs, n_sums = scenes.flight_requests(world, [[3000.0, 3000.0]])
    ctx = native.Context(0)
    dev = ctx.flight_boxes(world.boxes)
    bad = segs.copy()
    bad[0]["first"] = len(world.boxes)
    with pytest.raises(RuntimeError, match="segment 0 boxes"):
        dev.sums(points, hz, bad, n_sums)
    bad = segs.copy()
    bad[0]["sum"] = n_sums
    with pytest.raises(RuntimeError, match="segment 0 sum"):
        dev.sums(points, hz, bad, n_sums)
    with pytest.raises(RuntimeError, match="horizons"):
        dev.sums(points, hz[:100], segs, n_sums)
    far = segs.copy()
    far["weight"] = abi.FLIGHT_WEIGHT_FAR
    with pytest.raises(RuntimeError, match="coarse_m"):
        dev.sums(points, hz, far, n_sums)
    boxes = world.boxes[:4].copy()
    boxes[2]["levels_db"][1, 3] = np.nan
    with pytest.raises(RuntimeError, match="box 2 level"):
        ctx.flight_boxes(boxes)
    dev.close()
    ctx.close()


def test_config_square_lattice_against_a_sample(world):
    """The full square of the flight workload (2000 flights, 1024^2 cells at 100 m) asked at a
    32 x 32 lattice: classes sum to the energy, and 24 of the points match the oracle."""
    full = scenes.flight_boxes_square()
    xs = np.linspace(1600.0, full.side_m - 1600.0, 32)
    xy = np.stack(np.meshgrid(xs, xs), -1).reshape(-1, 2)
    points, hz, segs, n_sums = scenes.flight_requests(full, xy)
    ctx = native.Context(0)
    dev = ctx.flight_boxes(full.boxes)
    got, st = dev.sums(points, hz, segs, n_sums, stats=True)
    energy = got[:, :abi.PERIODS]
    classes = got[:, abi.PERIODS:abi.PERIODS * (1 + abi.PASS_CLASSES)].reshape(n_sums, abi.PERIODS, -1).sum(-1)
    assert np.allclose(classes, energy, rtol=1e-12, atol=0.0)
    pick = np.random.default_rng(41).choice(len(points), 24, replace=False)
    mine = np.isin(segs["point"], pick)
    want, _ = oracle.flight_sums(full.boxes, points, hz, segs[mine], n_sums)
    sums = np.concatenate([2 * pick, 2 * pick + 1])
    _compare(got[sums], want[sums], "config square")
    print(f"config square: {len(full.boxes)} boxes, {st['box_reads']} reads, {st['boxes_heard']} heard, "
          f"{st['kernel_ms']:.1f} ms, {st['box_reads'] / st['kernel_ms'] / 1e6:.2f} G reads/s")
    dev.close()
    ctx.close()
