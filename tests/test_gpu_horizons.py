"""The points' horizons for aircraft screening built on the device (qm_scene_flight_horizons) against
the oracle's restatement of Horizons::build (popup/src/aircraft/horizons.rs:145-198) on the same
scene: terrain sampled in 32 sectors, a 512 m building ray in each of 256 sectors through the f64
crossing walk, laid out as write_f32 lays them out. Empty bands agree exactly and every float within
1e-5 relative (the sector directions' sines and cosines are the device's and the C library's); the
horizons then screen the same boxes alike."""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu


def _points(scene, ora, rng, n):
    ext = np.array(scene.extent_steps, dtype=np.float64)
    xy = rng.uniform(0.1, 0.9, (n, 2)) * ext
    xy[: n // 2] = np.round(xy[: n // 2])  # lattice points and fractional ones
    own = ora.enclosing(np.round(xy).astype(np.int64))
    own[n // 2:] = 0  # a fractional point stands in nothing by its own right
    ground = np.array([ora.profile(p, p)[2][0] for p in np.round(xy).astype(np.int64)])
    return xy, ground + rng.uniform(2.0, 30.0, n), own


@pytest.mark.parametrize("which", ["terrain", "road"])
def test_device_horizons_match_the_oracle(which):
    scene = scenes.terrain_square(scale=0.125)[0] if which == "terrain" else scenes.road_square()[0]
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(71)
    xy, alt, own = _points(scene, ora, rng, 48)
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    got = dev.flight_horizons(xy, alt, own)
    want = ora.flight_horizons(xy, alt, own)
    assert np.array_equal(np.isnan(got), np.isnan(want))
    # A sector without any edge keeps -inf as its steepest tangent, alike on both sides.
    infinite = np.isinf(want)
    assert np.array_equal(got[infinite], want[infinite]) and not np.isinf(got[~infinite]).any()
    ok = np.isfinite(want)
    scale = np.maximum(np.abs(want[ok]), 1e-6)
    err = np.abs(got[ok] - want[ok]) / scale
    assert err.max() < 1e-5, float(err.max())
    inside = int((own != 0).sum())
    print(f"{which}: {len(xy)} points ({inside} inside buildings), {int(ok.sum())} floats set, "
          f"max relative difference {err.max():.1e}")
    dev.close()
    ctx.close()


def test_device_horizons_screen_boxes_as_the_oracles_do():
    scene = scenes.terrain_square(scale=0.125)[0]
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(73)
    xy, alt, own = _points(scene, ora, rng, 8)
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    hz_dev = dev.flight_horizons(xy, alt, own)
    hz_ora = ora.flight_horizons(xy, alt, own)
    world = scenes.flight_boxes_square(seed=13, n_flights=60, receivers=64)
    lattice = rng.uniform(500.0, world.side_m - 500.0, (8, 2))
    points, _, segs, n_sums = scenes.flight_requests(world, lattice, horizons=False)
    points["horizons"] = np.arange(8, dtype=np.uint64) * abi.HORIZON_FLOATS
    boxes = ctx.flight_boxes(world.boxes)
    a = boxes.sums(points, hz_dev.reshape(-1), segs, n_sums)
    b, _ = oracle.flight_sums(world.boxes, points, hz_ora.reshape(-1), segs, n_sums)
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-300)
    rel[b == 0] = np.abs(a[b == 0])
    assert rel.max() < 1e-6, float(rel.max())
    boxes.close()
    dev.close()
    ctx.close()


def test_bad_points_are_refused():
    scene = scenes.road_square()[0]
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    with pytest.raises(RuntimeError, match="point 1 position"):
        dev.flight_horizons([[10.0, 10.0], [np.nan, 3.0]], [4.0, 4.0], [0, 0])
    dev.close()
    ctx.close()


def test_flight_sums_on_the_scene_read_the_scenes_horizons():
    """qm_flight_sums_on_scene builds the horizons on the device and sums through them: the sums of
    qm_flight_sums given qm_scene_flight_horizons' floats from the host (the lattice step is a power
    of two, so the points' metres divide back to the same steps), up to the order in which the
    kernel's FP64 atomic additions land (1e-12 relative), and within the horizons' own 1e-5
    rounding of the oracle's sums through the oracle's horizons."""
    scene = scenes.terrain_square(scale=0.125)[0]
    ora = oracle.OracleScene(scene)
    rng = np.random.default_rng(79)
    xy, alt, own = _points(scene, ora, rng, 12)
    world = scenes.flight_boxes_square(seed=17, n_flights=80, receivers=64)
    points, _, segs, n_sums = scenes.flight_requests(world, xy * scene.step_m, horizons=False)
    points["altitude_m"] = alt
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    boxes = ctx.flight_boxes(world.boxes)
    got, st = boxes.sums_on_scene(dev, points, own, segs, n_sums, stats=True)
    assert np.frexp(scene.step_m)[0] == 0.5  # a power of two
    rows = points.copy()
    rows["horizons"] = np.arange(len(rows), dtype=np.uint64) * abi.HORIZON_FLOATS
    same = boxes.sums(rows, dev.flight_horizons(xy, alt, own).reshape(-1), segs, n_sums)
    assert np.array_equal(got != 0.0, same != 0.0)
    assert (np.abs(got - same) <= 1e-12 * np.abs(same)).all()
    hz = ora.flight_horizons(xy, alt, own)
    want, heard = oracle.flight_sums(world.boxes, rows, hz.reshape(-1), segs, n_sums)
    assert st["boxes_heard"] == heard > 0
    rel = np.abs(got - want) / np.maximum(np.abs(want), 1e-300)
    rel[want == 0] = np.abs(got[want == 0])
    assert rel.max() < 1e-6, float(rel.max())
    boxes.close()
    dev.close()
    ctx.close()
