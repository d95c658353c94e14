"""A scene built from an `obstacles` tile (qmobs2) through the library's reader paints like the
oracle: crossing lists bit for bit, cell levels within 0.05 dB."""

import numpy as np
import pytest

from quietmap_b200.physics import alpha_bands
from oracle import obstacles as ob
from oracle import oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu

TILE = ob.CELLS_PER_SIDE * ob.CELL_STEPS  # 32,768 steps a side; its centre is local 0


def _tile_outlines(rng):
    outlines = []
    for k in range(150):
        cx, cy = (int(v) for v in rng.integers(-4000, 4000, 2))
        w, h = (int(v) for v in rng.integers(150, 700, 2))
        outlines.append(dict(footprint_id=(0x0114_00AD << 32) | (2 * k), kind=ob.EXTERIOR, envelope=ob.RESIDENTIAL,
                             height_m=float(rng.integers(30, 250)) / 10.0,
                             vertices=[(cx, cy), (cx + w, cy), (cx + w, cy + h), (cx, cy + h), (cx, cy)]))
        if k % 10 == 0:  # a courtyard: a hole of the same footprint
            q = min(w, h) // 4
            outlines.append(dict(footprint_id=(0x0114_00AD << 32) | (2 * k), kind=ob.HOLE, envelope=ob.RESIDENTIAL,
                                 height_m=outlines[-1]["height_m"],
                                 vertices=[(cx + q, cy + q), (cx + w - q, cy + q), (cx + w - q, cy + h - q),
                                           (cx + q, cy + h - q), (cx + q, cy + q)]))
    for k in range(12):
        a = tuple(int(v) for v in rng.integers(-4500, 4500, 2))
        b = tuple(int(v) for v in rng.integers(-4500, 4500, 2))
        outlines.append(dict(footprint_id=(0x0114_00AE << 32) | k, kind=ob.WALL, envelope=ob.OUTDOOR,
                             height_m=3.0, vertices=[a, b]))
    outlines.sort(key=lambda o: o["footprint_id"])
    return outlines


def _scene(rng):
    data = ob.encode(_tile_outlines(rng))
    outlines, vertices, _ = native.obstacles_outlines(data, offset=(TILE // 2, TILE // 2))
    src = np.zeros(24, dtype=abi.SOURCE_DTYPE)
    src["x"] = TILE // 2 + rng.integers(-5000, 5000, 24)
    src["y"] = TILE // 2 + rng.integers(-5000, 5000, 24)
    src["height_m"] = 0.05
    src["ground_factor"] = -1.0
    src["energy"] = 10.0 ** 9.0
    return scenes.Scene(step_m=1.0 / 32.0, cell_steps=256, extent_steps=(TILE, TILE), vertices=vertices,
                        outlines=outlines, sources=src, favourable=np.zeros((3, 16)),
                        alpha_db_per_km=alpha_bands(15.0, 70.0), flat_altitude_m=0.0, flat_ground_factor=0.5,
                        name="obstacles tile")


def test_a_tile_scene_paints_like_the_oracle():
    rng = np.random.default_rng(31)
    scene = _scene(rng)
    ctx = native.Context(0)
    dev, ora = ctx.scene(scene), oracle.OracleScene(scene)
    frm = TILE // 2 + rng.integers(-5000, 5000, (400, 2))
    to = TILE // 2 + rng.integers(-5000, 5000, (400, 2))
    counts, edges, t, flags, status = dev.list_crossings(frm, to)
    assert not status.any()
    for i in range(len(frm)):
        ref = ora.crossings(frm[i], to[i])
        n = len(ref["t"])
        assert counts[i] == n
        np.testing.assert_array_equal(edges[i, :n], ref["edge"])
        np.testing.assert_array_equal(t[i, :n], ref["t"])
    grid = scenes.Grid(origin=(TILE // 2 - 4000, TILE // 2 - 4000), spacing=1000, nx=8, ny=8)
    _, dba, _, _, _ = dev.paint_grid(grid)
    e, _, _ = ora.paint_grid(grid)
    with np.errstate(divide="ignore"):
        ref = 10.0 * np.log10(e.sum(axis=1))
    np.testing.assert_allclose(dba, ref, atol=0.05)
    ctx.close()
