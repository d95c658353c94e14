"""Doc 29 flights on the GPU (qm_flight_grid) against the FP64 oracle on the same seeded flights."""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import native, scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    return native.Context(0)


def _compare(gpu, ref, cells=None):
    lae_g, thirds_g, sone_g = gpu
    lae_r, thirds_r, sone_r = ref
    if cells is not None:
        lae_g, thirds_g, sone_g = lae_g[cells], thirds_g[cells], sone_g[cells]
    heard = np.isfinite(lae_r)
    assert np.array_equal(heard, np.isfinite(lae_g))
    assert np.max(np.abs(lae_g[heard] - lae_r[heard])) <= 0.05
    assert np.max(np.abs(thirds_g[heard] - thirds_r[heard])) <= 0.05
    rel = np.abs(sone_g[heard] - sone_r[heard]) / np.maximum(sone_r[heard], 1e-3)
    assert np.max(rel) <= 0.005


def test_flight_grid_matches_oracle_small(ctx):
    f = scenes.flights_square(n_flights=120, receivers=64, spacing_m=400.0)
    _compare(ctx.flight_grid(f), oracle.flight_grid(f))


def test_flight_grid_culling_and_ragged_grid(ctx):
    # A grid that is no multiple of the 16 x 16 cell tile, with a reach that culls most flights.
    f = scenes.flights_square(seed=5, n_flights=60, receivers=40, spacing_m=900.0, reach_m=4000.0)
    f.grid["nx"], f.grid["ny"] = 37, 29
    _compare(ctx.flight_grid(f), oracle.flight_grid(f))


def test_flight_grid_far_ahead_and_behind_segments(ctx):
    # Receivers far along the line of long level segments: the finite-segment fraction is the
    # difference of two values near pi/2 there.
    f = scenes.flights_square(seed=6, n_flights=8, segments_per_flight=3, receivers=16, spacing_m=3000.0,
                              segment_m=4000.0, reach_m=0.0)
    f.segments["start"][:, 2] = 900.0
    f.segments["end"][:, 2] = 900.0
    _compare(ctx.flight_grid(f), oracle.flight_grid(f))


def test_flight_grid_full_size_sampled(ctx):
    # 1024^2 cells at 100 m, 2000 flights x 50 segments; the oracle checks a sample of cells.
    f = scenes.flights_square()
    gpu = ctx.flight_grid(f)
    rng = np.random.default_rng(11)
    cells = np.sort(rng.choice(1024 * 1024, 96, replace=False))
    ref = [oracle.flight_grid(f, int(c), int(c) + 1) for c in cells]
    ref = tuple(np.concatenate([r[i] for r in ref]) for i in range(3))
    _compare(gpu, ref, cells)
    # every cell is heard and its loudness is finite
    assert np.all(np.isfinite(gpu[0])) and np.all(np.isfinite(gpu[2]))


def test_flight_grid_rejects_bad_input(ctx):
    f = scenes.flights_square(n_flights=3, receivers=8)
    f.segments["power"][1] = 9.5
    with pytest.raises(native.QmError):
        ctx.flight_grid(f)
    f = scenes.flights_square(n_flights=3, receivers=8)
    f.segments["flight"][0] = 2  # not grouped by flight
    with pytest.raises(native.QmError):
        ctx.flight_grid(f)
