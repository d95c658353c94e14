"""The grid painter for callers that cannot allocate device memory (qm_paint_grid_static).

Such a caller (an engine that owns every device allocation, or a thread that may not allocate after
its set-up) gets the same painting as qm_paint_grid with every intermediate buffer carved out of the
library's static device array. This file is collected last so that a run stopping at its first
failure has already run every other test; it passes alone in a fresh process too (its first call
looks up the array's device address).
"""

import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from quietmap_b200 import abi, native, scenes

pytestmark = pytest.mark.gpu

TOL_DB = 0.05  # the parity tolerance of the painter tests


def _bind():
    L = native.lib()
    f = L.qm_paint_grid_static
    f.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), C.POINTER(C.c_float), C.POINTER(C.c_float),
                  C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.POINTER(abi.PaintStats)]
    f.restype = C.c_int
    return f


def _paint_static(f, dev, grid):
    g = abi.grid_desc(grid)
    bands = np.zeros((grid.cells, 8), np.float32)
    dba = np.zeros(grid.cells, np.float32)
    lden = np.zeros(grid.cells, np.float32)
    hist = np.zeros(grid.n_bins, np.uint32)
    stats = abi.PaintStats()
    status = f(dev.handle, C.byref(g), abi.ptr(bands, C.c_float), abi.ptr(dba, C.c_float), abi.ptr(lden, C.c_float),
               abi.ptr(hist, C.c_uint32), C.byref(stats))
    return status, bands, dba, lden, hist, stats


def test_static_scratch_painter_matches_the_allocating_one_on_two_calls():
    f = _bind()
    scene, full = scenes.road_square()
    grid = scenes.Grid(origin=full.origin, spacing=full.spacing, nx=64, ny=32)
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    ref_bands, ref_dba, ref_lden, ref_hist, ref_stats = dev.paint_grid(grid)
    runs = []
    for _ in range(2):
        status, bands, dba, lden, hist, stats = _paint_static(f, dev, grid)
        assert status == abi.QM_OK, native.lib().qm_last_error(ctx.handle)
        assert stats.paths == ref_stats["paths"] and stats.failed_paths == 0
        np.testing.assert_allclose(dba, ref_dba, atol=TOL_DB)
        np.testing.assert_allclose(lden, ref_lden, atol=TOL_DB)
        ok = np.isfinite(ref_bands)
        np.testing.assert_allclose(bands[ok], ref_bands[ok], atol=TOL_DB)
        # Exact counts of its own levels under the reference's bin rule.
        np.testing.assert_array_equal(
            hist, oracle.level_histogram(dba.astype(np.float64), grid.level_min_db, grid.bin_db, grid.n_bins))
        runs.append((bands, dba, lden, hist))
    # The second call starts from cleared buffers: the same answer bit for bit.
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)
    dev.close()
    ctx.close()


def test_static_scratch_painter_rejects_grids_beyond_its_limit():
    f = _bind()
    scene, full = scenes.road_square(n_roads=4, n_buildings=4)
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    grid = scenes.Grid(origin=(0, 0), spacing=1, nx=300, ny=300)  # 90,000 cells > 65,536
    status, *_ = _paint_static(f, dev, grid)
    assert status == abi.QM_ERR_CAPACITY
    assert b"65536" in native.lib().qm_last_error(ctx.handle)
    dev.close()
    ctx.close()


def test_static_scratch_painter_sets_up_receivers_as_the_host_does_on_terrain():
    """On a DEM with grid receivers inside buildings: the device set-up's altitudes and own
    footprints must be those of qm_paint_grid's host set-up, or the levels would differ (a receiver
    inside a building hears through its own walls only when it knows them as its own)."""
    f = _bind()
    scene, _ = scenes.terrain_square(scale=0.125)
    # A 32 x 32 grid at 1 m around the first building's first vertex.
    v = scene.vertices[scene.outlines[0]["first_vertex"]]
    spacing = int(round(1.0 / scene.step_m))
    grid = scenes.Grid(origin=(int(v[0]) - 16 * spacing, int(v[1]) - 16 * spacing), spacing=spacing, nx=32, ny=32)
    ora = oracle.OracleScene(scene)
    inside = ora.enclosing(grid.receiver_xy())
    assert np.count_nonzero(inside) > 0
    ctx = native.Context(0)
    dev = ctx.scene(scene)
    ref_bands, ref_dba, ref_lden, _, ref_stats = dev.paint_grid(grid)
    assert ref_stats["failed_paths"] == 0
    for _ in range(2):
        status, bands, dba, lden, hist, stats = _paint_static(f, dev, grid)
        assert status == abi.QM_OK, native.lib().qm_last_error(ctx.handle)
        np.testing.assert_allclose(dba, ref_dba, atol=TOL_DB)
        np.testing.assert_allclose(lden, ref_lden, atol=TOL_DB)
        ok = np.isfinite(ref_bands)
        np.testing.assert_allclose(bands[ok], ref_bands[ok], atol=TOL_DB)
    dev.close()
    ctx.close()
