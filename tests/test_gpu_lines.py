"""Line pieces as candidates of Batch::evaluate on the device (qm_scene_line_pieces, qm_evaluate_pairs)
against the oracle's evaluation of a whole piece (qmo_line_piece: the reference's quadrature, the
receiver's skyline, each node's ray from its point along the piece by the f64 walks).

Pieces of 20-200 m with fractional ends on the scaled terrain square (DEM, buildings) and on the
flat road square; every pair's PairEnergy (mixed, calm and downwind per period) within 0.05 dB of
the oracle at the maximum.
"""

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu

TOL_DB = 0.05


def _pieces(scene, rng, n):
    ext = np.array(scene.extent_steps, dtype=np.float64)
    out = np.zeros(n, dtype=abi.LINE_SOURCE_DTYPE)
    for k in range(n):
        a = rng.uniform(0.05, 0.95, 2) * ext
        angle = rng.uniform(0.0, 2.0 * np.pi)
        length = rng.uniform(20.0, 200.0) / scene.step_m
        b = np.clip(a + length * np.array([np.cos(angle), np.sin(angle)]), 1.0, ext - 2.0)
        out[k]["a"], out[k]["b"] = a, b
        src = out[k]["source"]
        src["height_m"] = 0.05 if k % 3 else 0.5
        src["ground_factor"] = -1.0
        src["layer"] = k % 2
        src["energy"][:] = 10.0 ** (rng.uniform(60.0, 90.0, (3, 8)) / 10.0)
    return out


@pytest.mark.parametrize("which", ["terrain", "road"])
def test_line_pieces_match_the_oracle(which):
    scene = scenes.terrain_square(scale=0.125)[0] if which == "terrain" else scenes.road_square()[0]
    rng = np.random.default_rng(61)
    pieces = _pieces(scene, rng, 24)
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    dev.line_pieces(pieces)
    ora = oracle.OracleScene(scene)
    ext = np.array(scene.extent_steps)
    n_rcv = 16
    rxy = rng.integers(1, ext - 1, (n_rcv, 2))
    own = ora.enclosing(rxy)
    pairs = [(r, k) for r in range(n_rcv) for k in rng.choice(len(pieces), 6, replace=False)]
    rop = np.array([r for r, _ in pairs], np.uint32)
    sop = np.array([len(scene.sources) + k for _, k in pairs], np.uint32)
    sums, bands, status, _ = dev.evaluate_pairs(rxy * scene.step_m, np.full(n_rcv, 4.0), own,
                                                np.arange(n_rcv, dtype=np.uint32), sop, rop, None, n_rcv)
    assert not status.any()
    ground = np.array([ora.profile(p, p)[2][0] for p in rxy])
    worst, nodes = 0.0, 0
    for i, (r, k) in enumerate(pairs):
        want_bands, want_states, n = ora.line_piece(rxy[r], ground[r] + 4.0, pieces[k]["a"], pieces[k]["b"],
                                                    pieces[k]["source"], own_footprint=int(own[r]))
        nodes += n
        want = np.concatenate([want_bands.sum(axis=1), want_states[0], want_states[1]])
        with np.errstate(divide="ignore"):
            got_db, want_db = 10.0 * np.log10(sums[i].astype(np.float64)), 10.0 * np.log10(want)
        assert np.array_equal(np.isfinite(got_db), np.isfinite(want_db)), (i, sums[i], want)
        heard = np.isfinite(want_db)
        err = np.abs(got_db[heard] - want_db[heard])
        worst = max(worst, float(err.max(initial=0.0)))
        assert err.max(initial=0.0) < TOL_DB, (i, r, k, got_db, want_db)
        b_db = 10.0 * np.log10(np.maximum(bands[i].astype(np.float64), 1e-300))
        wb_db = 10.0 * np.log10(np.maximum(want_bands, 1e-300))
        ok = want_bands > want_bands.max() * 1e-6
        assert np.abs(b_db[ok] - wb_db[ok]).max(initial=0.0) < TOL_DB, (i, r, k)
    print(f"{which}: {len(pairs)} line pairs, {nodes} quadrature nodes, max |error| {worst:.2e} dB")
    dev.close()
    ctx.close()
