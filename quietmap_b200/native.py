"""ctypes binding of the CUDA library (quietmap_b200/libqm_b200.so, C ABI of include/qm_batch.h).

There is no CPU fallback: if the library is missing or no sm_100 device is present, every call
raises. The library is built in-tree by quietmap_b200/build.py (or `__graft_entry__.build()`).
"""

import ctypes as C
import math
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqm_b200.so")

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_U32 = C.POINTER(C.c_uint32)
_U64 = C.POINTER(C.c_uint64)
_I32 = C.POINTER(C.c_int32)
_U8 = C.POINTER(C.c_uint8)


class QmError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"qm status {status}: {message}")
        self.status = status


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QmError(abi.QM_ERR_UNSUPPORTED,
                          f"{LIB_PATH} is missing: build it with quietmap_b200/build.py")
        L = C.CDLL(LIB_PATH)
        L.qm_abi_version.restype = C.c_int
        L.qm_open.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.qm_open.restype = C.c_int
        L.qm_close.argtypes = [C.c_void_p]
        L.qm_last_error.argtypes = [C.c_void_p]
        L.qm_last_error.restype = C.c_char_p
        L.qm_scene_upload.argtypes = [C.c_void_p, C.POINTER(abi.SceneDesc), C.POINTER(C.c_void_p)]
        L.qm_scene_upload.restype = C.c_int
        L.qm_scene_free.argtypes = [C.c_void_p]
        L.qm_evaluate_pairs.argtypes = [C.c_void_p, _D, _F, _U64, _U32, C.c_size_t, _U32, _U32, _F, C.c_size_t,
                                        _F, _F, _U32, _F, C.c_size_t]
        L.qm_evaluate_pairs.restype = C.c_int
        L.qm_scene_line_pieces.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t]
        L.qm_scene_line_pieces.restype = C.c_int
        L.qm_paint_grid.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), _F, _F, _F, _U32,
                                    C.POINTER(abi.PaintStats)]
        L.qm_paint_grid.restype = C.c_int
        L.qm_zwicker.argtypes = [C.c_void_p, _F, C.c_size_t, _F]
        L.qm_check_bounded_wait.argtypes = [C.c_void_p, C.c_double, _D]
        L.qm_check_bounded_wait.restype = C.c_int
        L.qm_zwicker.restype = C.c_int
        L.qm_level_histogram.argtypes = [C.c_void_p, _F, C.c_size_t, C.c_double, C.c_double, C.c_uint32, _U32]
        L.qm_level_histogram.restype = C.c_int
        L.qm_quantize_cells.argtypes = [C.c_void_p, _D, _D, _U8, C.c_size_t, _U8, _U8]
        L.qm_quantize_cells.restype = C.c_int
        L.qm_hm3_predict.argtypes = [C.c_void_p, _U8, _U8, C.c_size_t, C.c_int, _U8]
        L.qm_hm3_predict.restype = C.c_int
        L.qm_line_level_table.argtypes = [C.POINTER(C.c_float)]
        L.qm_line_level_table.restype = C.c_int
        L.qm_line_level_quantiles.argtypes = [C.c_void_p, _D, _D, C.c_size_t, _D]
        L.qm_line_level_quantiles.restype = C.c_int
        L.qm_hm3_unpredict.argtypes = [_U8, C.c_size_t, C.c_uint32, C.c_int, _U8]
        L.qm_hm3_unpredict.restype = C.c_int
        L.qm_obstacles_check.argtypes = [_U8, C.c_size_t, C.POINTER(abi.ObstaclesCounts)]
        L.qm_obstacles_check.restype = C.c_int
        L.qm_obstacles_outlines.argtypes = [_U8, C.c_size_t, C.c_int32, C.c_int32, C.c_uint32, C.c_void_p,
                                            _I32, _U8]
        L.qm_obstacles_outlines.restype = C.c_int
        L.qm_obstacles_merge.argtypes = [C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), _I32, C.c_size_t, C.c_void_p,
                                         _U32, _I32, _U32, _U8]
        L.qm_obstacles_merge.restype = C.c_int
        L.qm_obstacles_cell_runs.argtypes = [_U8, C.c_size_t, C.c_uint32, C.c_uint32, _U32, C.c_uint32, _U32]
        L.qm_obstacles_cell_runs.restype = C.c_int
        L.qm_terrain_decode.argtypes = [_U8, C.c_size_t, C.POINTER(abi.TerrainWindow), C.POINTER(C.c_uint16), _U8,
                                        _U8, _U8]
        L.qm_terrain_decode.restype = C.c_int
        L.qm_terrain_fine_decode.argtypes = [_U8, C.c_size_t, C.POINTER(abi.TerrainWindow), C.POINTER(C.c_int16)]
        L.qm_terrain_fine_decode.restype = C.c_int
        L.qm_mercator_from_degrees.argtypes = [C.c_double, C.c_double, _D, _D]
        L.qm_mercator_from_degrees.restype = None
        L.qm_terrain_window_of_tile.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(abi.TerrainWindow)]
        L.qm_terrain_window_of_tile.restype = C.c_int
        L.qm_terrain_column_of.argtypes = [C.POINTER(abi.TerrainWindow), C.c_double]
        L.qm_terrain_column_of.restype = C.c_double
        L.qm_terrain_sample.argtypes = [C.POINTER(abi.TerrainWindow), C.POINTER(C.c_uint16), _U8, _U8, _U8, _D,
                                        C.c_size_t, C.POINTER(abi.GroundSample), _U8]
        L.qm_terrain_sample.restype = C.c_int
        L.qm_weather_place.argtypes = [_U8, C.c_size_t, C.c_double, C.c_double, _D, _D]
        L.qm_weather_place.restype = C.c_int
        L.qm_weather_read_place.argtypes = [C.c_char_p, C.c_double, C.c_double, _D, _D]
        L.qm_weather_read_place.restype = C.c_int
        L.qm_list_crossings.argtypes = [C.c_void_p, _I32, _I32, C.c_size_t, C.c_uint32, _U32, _U32, _D, _U32, _U32]
        L.qm_list_crossings.restype = C.c_int
        L.qm_flight_grid.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t,
                                     C.POINTER(abi.FlightGridDesc), _F, _F, _F, C.POINTER(abi.FlightStats)]
        L.qm_flight_grid.restype = C.c_int
        P = C.POINTER(C.c_void_p)
        L.qm_surrogate_create.argtypes = [C.c_void_p, _F, P]
        L.qm_surrogate_create.restype = C.c_int
        L.qm_surrogate_free.argtypes = [C.c_void_p]
        L.qm_surrogate_set_kernel.argtypes = [C.c_void_p, C.c_int]
        L.qm_surrogate_set_kernel.restype = C.c_int
        L.qm_surrogate_params.argtypes = [C.c_void_p, _F]
        L.qm_surrogate_params.restype = C.c_int
        L.qm_surrogate_samples.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), _F, _F, C.POINTER(C.c_uint8)]
        L.qm_surrogate_samples.restype = C.c_int
        L.qm_surrogate_forward.argtypes = [C.c_void_p, _F, C.c_size_t, _F]
        L.qm_surrogate_forward.restype = C.c_int
        L.qm_surrogate_gradients.argtypes = [C.c_void_p, _F, _F, C.c_size_t, _F, _D]
        L.qm_surrogate_gradients.restype = C.c_int
        L.qm_surrogate_train.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(abi.GridDesc), C.c_size_t,
                                         C.POINTER(abi.TrainConfig), _D, _U64]
        L.qm_surrogate_train.restype = C.c_int
        L.qm_paint_grid_surrogate.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), C.c_void_p, _F, _F, _F, _U32,
                                              C.POINTER(abi.PaintStats), _U64]
        L.qm_paint_grid_surrogate.restype = C.c_int
        L.qm_tile_bucket.argtypes = [C.POINTER(abi.TileDesc)]
        L.qm_tile_bucket.restype = C.c_uint32
        L.qm_tune_default.argtypes = [C.POINTER(abi.TuneTable)]
        L.qm_batch_autotune.argtypes = [C.c_void_p, C.POINTER(abi.TileDesc), C.c_size_t, C.POINTER(abi.TuneTable), _F]
        L.qm_batch_autotune.restype = C.c_int
        L.qm_batch_plan_create.argtypes = [C.c_void_p, C.POINTER(abi.TileDesc), C.c_size_t, C.c_uint64,
                                           C.POINTER(abi.TuneTable), C.c_uint32, P]
        L.qm_batch_plan_create.restype = C.c_int
        L.qm_batch_plan_free.argtypes = [C.c_void_p]
        L.qm_batch_plan_run.argtypes = [C.c_void_p, C.POINTER(abi.PaintStats)]
        L.qm_batch_plan_run.restype = C.c_int
        L.qm_batch_plan_read.argtypes = [C.c_void_p, _F, _F, _F]
        L.qm_batch_plan_read.restype = C.c_int
        L.qm_line_quadrature_nodes.argtypes = [_D, _D, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                               C.POINTER(C.c_size_t), C.POINTER(abi.LinePieceInfo)]
        L.qm_line_quadrature_nodes.restype = C.c_int
        L.qm_skyline_build.argtypes = [C.POINTER(C.c_int32), C.c_size_t, C.c_void_p, C.c_size_t, C.c_double,
                                       C.POINTER(C.c_void_p)]
        L.qm_skyline_build.restype = C.c_int
        L.qm_skyline_counts.argtypes = [C.c_void_p, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
        L.qm_skyline_counts.restype = C.c_int
        L.qm_skyline_arcs.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double,
                                      C.c_double, _D, C.c_size_t, C.POINTER(C.c_size_t)]
        L.qm_skyline_arcs.restype = C.c_int
        L.qm_skyline_free.argtypes = [C.c_void_p]
        L.qm_skyline_free.restype = None
        L.qm_distribution_bins.argtypes = [C.c_double, C.POINTER(C.c_size_t)]
        L.qm_distribution_bins.restype = C.c_int
        L.qm_distribution_with_line.argtypes = [C.c_double, _D, C.c_double, _D, C.c_size_t, C.c_double, _D, _D]
        L.qm_distribution_with_line.restype = C.c_int
        L.qm_distribution_exceeded_db.argtypes = [C.c_double, _D, C.c_double, _D]
        L.qm_distribution_exceeded_db.restype = C.c_int
        L.qm_distribution_line_values.argtypes = [C.c_double, C.c_double, _D, C.c_size_t, C.POINTER(C.c_size_t)]
        L.qm_distribution_line_values.restype = C.c_int
        L.qm_distribution_pass_values.argtypes = [C.c_double, _D, C.c_size_t, C.POINTER(C.c_size_t)]
        L.qm_distribution_pass_values.restype = C.c_int
        L.qm_distribution_layers.argtypes = [C.c_double, C.c_void_p, C.c_size_t, _D, C.c_size_t, _D, _D, _D, _D]
        L.qm_distribution_layers.restype = C.c_int
        L.qm_distribution_percentiles.argtypes = [C.c_double, _D, _D]
        L.qm_distribution_percentiles.restype = C.c_int
        L.qm_pixel_ndens.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.c_uint32, C.c_double, _D, C.c_size_t, _U32,
                                     _D, _D]
        L.qm_pixel_ndens.restype = C.c_int
        L.qm_pixel_loudness.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_size_t, _U64, C.c_size_t, C.c_uint32,
                                        C.c_double, _D, C.c_size_t, _U32, _F, _D]
        L.qm_pixel_loudness.restype = C.c_int
        L.qm_scene_flight_horizons.argtypes = [C.c_void_p, _D, _D, _U64, C.c_size_t, _F, _D]
        L.qm_flight_sums_on_scene.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _U64, C.c_size_t, C.c_void_p,
                                              C.c_size_t, _D, C.c_size_t, C.POINTER(abi.FlightSumsStats)]
        L.qm_flight_sums_on_scene.restype = C.c_int
        L.qm_scene_flight_horizons.restype = C.c_int
        L.qm_flight_boxes_upload.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p)]
        L.qm_flight_boxes_upload.restype = C.c_int
        L.qm_flight_boxes_free.argtypes = [C.c_void_p]
        L.qm_flight_boxes_free.restype = None
        L.qm_flight_sums.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, _F, C.c_size_t, C.c_void_p,
                                     C.c_size_t, _D, C.c_size_t, C.POINTER(abi.FlightSumsStats)]
        L.qm_flight_sums.restype = C.c_int
        L.qm_pixel_distributions.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.c_uint32, C.c_double, _D, C.c_size_t,
                                             _U32, _D, _D, _D, _D]
        L.qm_pixel_distributions.restype = C.c_int
        L.qm_hour_groups.argtypes = [_D, C.c_size_t, C.c_uint32, C.c_uint32, _U32, _U32, _D, C.POINTER(C.c_size_t)]
        L.qm_hour_groups.restype = C.c_int
        L.qm_distribution_state_means.argtypes = [_D, _D, C.c_size_t, _D, _D]
        L.qm_distribution_state_means.restype = C.c_int
        L.qm_pixel_read.argtypes = [C.POINTER(C.c_float), C.c_size_t, C.c_uint32, C.c_uint32, C.c_void_p,
                                    C.POINTER(C.c_int32), C.c_size_t, C.POINTER(C.c_size_t), _D, _D, _U8]
        L.qm_pixel_read.restype = C.c_int
        L.qm_loudness_curve_shape.argtypes = [_D, _D, C.POINTER(C.c_int)]
        L.qm_loudness_curve_shape.restype = C.c_int
        L.qm_distribution_loudness.argtypes = [C.c_double, _D, _D, _D, _D]
        L.qm_distribution_loudness.restype = C.c_int
        L.qm_distribution_merge_states.argtypes = [C.c_void_p, C.c_size_t, C.c_double]
        L.qm_distribution_merge_states.restype = C.c_int
        L.qm_distribution_layers_grouped.argtypes = [C.c_double, C.c_void_p, C.c_size_t, _D, C.c_size_t, C.c_uint32,
                                                     _U32, C.c_size_t, _D, _U8, _D, _D, _D, _D]
        L.qm_distribution_layers_grouped.restype = C.c_int
        if L.qm_abi_version() != abi.ABI_VERSION:
            raise QmError(abi.QM_ERR_UNSUPPORTED, "library ABI version mismatch")
        _lib = L
    return _lib


def _check(status, ctx=None):
    if status != abi.QM_OK:
        message = lib().qm_last_error(ctx).decode(errors="replace")
        raise QmError(status, message)


class DeviceFlightBoxes:
    """A square's aircraft boxes decoded once on the device (qm_flight_boxes_upload); `sums` runs
    Batch::flight_sums over them (qm_flight_sums)."""

    def __init__(self, ctx, boxes):
        self.ctx = ctx
        b = np.ascontiguousarray(boxes, dtype=abi.FLIGHT_BOX_DTYPE)
        self.n = len(b)
        self.handle = C.c_void_p()
        _check(lib().qm_flight_boxes_upload(ctx.handle, b.ctypes.data if len(b) else None, len(b),
                                            C.byref(self.handle)), ctx.handle)

    def sums(self, points, horizons, segments, n_sums, stats=False):
        """sums [n_sums][FLIGHT_SUMS] of every request band, and a dict of work and device time
        when `stats`."""
        p = np.ascontiguousarray(points, dtype=abi.FLIGHT_POINT_DTYPE)
        h = None if horizons is None else np.ascontiguousarray(horizons, dtype=np.float32)
        s = np.ascontiguousarray(segments, dtype=abi.BOX_SEGMENT_DTYPE)
        out = np.zeros((n_sums, abi.FLIGHT_SUMS))
        st = abi.FlightSumsStats()
        _check(lib().qm_flight_sums(self.ctx.handle, self.handle, p.ctypes.data if len(p) else None, len(p),
                                    None if h is None else abi.ptr(h, C.c_float), 0 if h is None else len(h),
                                    s.ctypes.data if len(s) else None, len(s), abi.ptr(out, C.c_double), n_sums,
                                    C.byref(st)), self.ctx.handle)
        if stats:
            return out, dict(box_reads=st.box_reads, boxes_heard=st.boxes_heard, kernel_ms=st.kernel_ms)
        return out

    def sums_on_scene(self, device_scene, points, own_footprint, segments, n_sums, stats=False):
        """`sums` with the points' horizons built and read on the device from `device_scene`
        (qm_flight_sums_on_scene); the points' positions in the square's metres."""
        p = np.ascontiguousarray(points, dtype=abi.FLIGHT_POINT_DTYPE)
        own = None if own_footprint is None else np.ascontiguousarray(own_footprint, dtype=np.uint64)
        s = np.ascontiguousarray(segments, dtype=abi.BOX_SEGMENT_DTYPE)
        out = np.zeros((n_sums, abi.FLIGHT_SUMS))
        st = abi.FlightSumsStats()
        _check(lib().qm_flight_sums_on_scene(device_scene.handle, self.handle, p.ctypes.data if len(p) else None,
                                             None if own is None else abi.ptr(own, C.c_uint64), len(p),
                                             s.ctypes.data if len(s) else None, len(s), abi.ptr(out, C.c_double),
                                             n_sums, C.byref(st)), self.ctx.handle)
        if stats:
            return out, dict(box_reads=st.box_reads, boxes_heard=st.boxes_heard, kernel_ms=st.kernel_ms)
        return out

    def close(self):
        if self.handle:
            lib().qm_flight_boxes_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One device (qm_open)."""

    def __init__(self, device=0):
        self.handle = C.c_void_p()
        _check(lib().qm_open(device, C.byref(self.handle)))

    def close(self):
        if self.handle:
            lib().qm_close(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def scene(self, scene):
        return DeviceScene(self, scene)

    def zwicker(self, thirds_db):
        thirds = np.ascontiguousarray(np.asarray(thirds_db, dtype=np.float32).reshape(-1, abi.THIRDS))
        out = np.zeros(len(thirds), np.float32)
        _check(lib().qm_zwicker(self.handle, abi.ptr(thirds, C.c_float), len(thirds), abi.ptr(out, C.c_float)),
               self.handle)
        return out

    def pixel_loudness(self, pixels, n_layers, bin_db=2.0, shares=None, runs=None, stats=False):
        """Batch::loudness on the device (qm_pixel_loudness): Nden per layer and for the place
        [n][n_layers + 1] of packed pixels (a list of float32 arrays, laid end to end), and the
        kernel's device time in ms when `stats`."""
        sizes = [len(p) for p in pixels]
        offsets = np.ascontiguousarray(np.concatenate([[0], np.cumsum(sizes)[:-1]]) if sizes else [], dtype=np.uint64)
        f = np.ascontiguousarray(np.concatenate(pixels) if pixels else np.zeros(0), dtype=np.float32)
        sh = np.ascontiguousarray(np.zeros((0, 24)) if shares is None else shares, dtype=np.float64).reshape(-1, 24)
        ru = None if runs is None else np.ascontiguousarray(runs, dtype=np.uint32)
        out = np.zeros((len(pixels), n_layers + 1), np.float32)
        ms = C.c_double(0.0)
        _check(lib().qm_pixel_loudness(self.handle, abi.ptr(f, C.c_float) if len(f) else None, len(f),
                                       abi.ptr(offsets, C.c_uint64) if len(offsets) else None, len(pixels),
                                       int(n_layers), float(bin_db), abi.ptr(sh, C.c_double) if len(sh) else None,
                                       len(sh), None if ru is None else abi.ptr(ru, C.c_uint32),
                                       abi.ptr(out, C.c_float), C.byref(ms)), self.handle)
        return (out, ms.value) if stats else out

    def flight_grid(self, flights, grid=None, sone=True, stats=False):
        """Doc 29 flights over a receiver grid: (LAE [cells], thirds [cells][28], sone [cells]),
        and a dict of work and device times when `stats`."""
        g = abi.flight_grid_desc(grid or flights.grid)
        cells = g.nx * g.ny
        types = np.ascontiguousarray(flights.types, dtype=abi.AIRCRAFT_TYPE_DTYPE)
        segs = np.ascontiguousarray(flights.segments, dtype=abi.FLIGHT_SEGMENT_DTYPE)
        lae = np.zeros(cells, np.float32)
        thirds = np.zeros((cells, abi.THIRDS), np.float32)
        out_sone = np.zeros(cells, np.float32) if sone else None
        st = abi.FlightStats()
        _check(lib().qm_flight_grid(self.handle, types.ctypes.data, len(types), segs.ctypes.data, len(segs),
                                    C.byref(g), abi.ptr(lae, C.c_float), abi.ptr(thirds, C.c_float),
                                    abi.ptr(out_sone, C.c_float) if sone else None, C.byref(st)), self.handle)
        if stats:
            return lae, thirds, out_sone, dict(pairs=st.pairs, pairs_in_reach=st.pairs_in_reach,
                                               kernel_ms=st.kernel_ms, loudness_ms=st.loudness_ms)
        return lae, thirds, out_sone

    def check_bounded_wait(self, limit_ms=1000.0):
        """The bounded wait's own check (qm_check_bounded_wait): the device time (ms) a wait on an
        mbarrier that nothing completes took to give up."""
        ms = C.c_double(0.0)
        _check(lib().qm_check_bounded_wait(self.handle, float(limit_ms), C.byref(ms)), self.handle)
        return ms.value

    def flight_boxes(self, boxes):
        """A square's aircraft boxes on the device (qm_flight_boxes_upload)."""
        return DeviceFlightBoxes(self, boxes)

    def quantize_cells(self, lden_energy, sone=None, assessed=None):
        """Map cells of pixels (qm_quantize_cells): (lden_cells [n][7], nden_cells [n][7] or None)
        from linear Lden energies [n][6], loudness [n][7] (sone) and assessed flags [n]."""
        energy = np.ascontiguousarray(np.asarray(lden_energy, dtype=np.float64).reshape(-1, abi.LAYERS))
        n = len(energy)
        s = None if sone is None else np.ascontiguousarray(np.asarray(sone, dtype=np.float64).reshape(n, abi.LAYERS + 1))
        a = None if assessed is None else np.ascontiguousarray(np.asarray(assessed, dtype=np.uint8).reshape(n))
        lc = np.zeros((n, abi.LAYERS + 1), np.uint8)
        nc = None if s is None else np.zeros((n, abi.LAYERS + 1), np.uint8)
        _check(lib().qm_quantize_cells(self.handle, abi.ptr(energy, C.c_double), abi.ptr(s, C.c_double),
                                       abi.ptr(a, C.c_uint8), n, abi.ptr(lc, C.c_uint8), abi.ptr(nc, C.c_uint8)),
               self.handle)
        return lc, nc

    def hm3_predict(self, cells, layers, metric):
        """HM3 / HMD tile streams before Brotli (qm_hm3_predict): cells [n][512][512] uint8,
        layers [n], metric 0 (loudness) or 1 (Lden) -> streams [n][6 + 512 * 512]."""
        c = np.ascontiguousarray(np.asarray(cells, dtype=np.uint8).reshape(-1, abi.HM3_TILE_PX * abi.HM3_TILE_PX))
        lay = np.ascontiguousarray(np.asarray(layers, dtype=np.uint8).reshape(len(c)))
        out = np.zeros((len(c), abi.HM3_STREAM_BYTES), np.uint8)
        _check(lib().qm_hm3_predict(self.handle, abi.ptr(c, C.c_uint8), abi.ptr(lay, C.c_uint8), len(c), int(metric),
                                    abi.ptr(out, C.c_uint8)), self.handle)
        return out

    def line_level_quantiles(self, lam, p):
        """The intensity, relative to its mean, a line of `lam` emitters per distance stays below
        with probability p, on the device (qm_line_level_quantiles); arrays broadcast together."""
        lam_b, p_b = np.broadcast_arrays(np.asarray(lam, dtype=np.float64), np.asarray(p, dtype=np.float64))
        lam_c, p_c = np.ascontiguousarray(lam_b.ravel()), np.ascontiguousarray(p_b.ravel())
        out = np.zeros(lam_c.size)
        _check(lib().qm_line_level_quantiles(self.handle, abi.ptr(lam_c, C.c_double), abi.ptr(p_c, C.c_double),
                                             lam_c.size, abi.ptr(out, C.c_double)), self.handle)
        return out.reshape(lam_b.shape)

    def level_histogram(self, levels_db, level_min_db=-30.0, bin_db=0.1, n_bins=1800):
        levels = np.ascontiguousarray(levels_db, dtype=np.float32).ravel()
        counts = np.zeros(n_bins, np.uint32)
        _check(lib().qm_level_histogram(self.handle, abi.ptr(levels, C.c_float), len(levels), level_min_db,
                                        bin_db, n_bins, abi.ptr(counts, C.c_uint32)), self.handle)
        return counts


def _tile_bytes(data):
    b = np.frombuffer(bytes(data), dtype=np.uint8)
    return b, abi.ptr(b, C.c_uint8) if len(b) else None


def line_level_table():
    """The library's line-level quantile table (qm_line_level_table): float32 [41][100]."""
    out = np.zeros((41, 100), np.float32)
    _check(lib().qm_line_level_table(abi.ptr(out, C.c_float)))
    return out


def hm3_unpredict(stream, layer, metric):
    """A decompressed HM3 / HMD stream back to its 512 x 512 cells (qm_hm3_unpredict), host only."""
    b, p = _tile_bytes(stream)
    cells = np.zeros((abi.HM3_TILE_PX, abi.HM3_TILE_PX), np.uint8)
    _check(lib().qm_hm3_unpredict(p, len(b), layer, metric, abi.ptr(cells, C.c_uint8)))
    return cells


def obstacles_check(data):
    """Checks an `obstacles` tile (qmobs2) and returns its header counts (qm_obstacles_check)."""
    b, p = _tile_bytes(data)
    counts = abi.ObstaclesCounts()
    _check(lib().qm_obstacles_check(p, len(b), C.byref(counts)))
    return {name: getattr(counts, name) for name in
            ("outlines", "vertices", "runs", "occupied_cells", "footprint_squares")}


def obstacles_outlines(data, offset=(0, 0), first_vertex_base=0):
    """A tile's outlines for a scene (qm_obstacles_outlines): (outlines [OUTLINE_DTYPE], vertices
    int32 [n][2] = the tile's int16 vertices + offset, envelope class codes uint8)."""
    counts = obstacles_check(data)
    b, p = _tile_bytes(data)
    outlines = np.zeros(counts["outlines"], abi.OUTLINE_DTYPE)
    vertices = np.zeros((counts["vertices"], 2), np.int32)
    envelope = np.zeros(counts["outlines"], np.uint8)
    _check(lib().qm_obstacles_outlines(p, len(b), int(offset[0]), int(offset[1]), first_vertex_base,
                                       outlines.ctypes.data if len(outlines) else None,
                                       abi.ptr(vertices, C.c_int32) if len(vertices) else None,
                                       abi.ptr(envelope, C.c_uint8) if len(envelope) else None))
    return outlines, vertices, envelope


def obstacles_merge(tiles, offsets):
    """Several tiles' outlines as one scene's (qm_obstacles_merge): each outline once, tiles at
    `offsets` (their centres in scene steps). Returns (outlines, vertices [n][2], envelope)."""
    arrays = [np.frombuffer(bytes(t), dtype=np.uint8) for t in tiles]
    ptrs = (C.c_void_p * len(arrays))(*[a.ctypes.data for a in arrays])
    sizes = (C.c_size_t * len(arrays))(*[len(a) for a in arrays])
    off = np.ascontiguousarray(np.asarray(offsets, dtype=np.int32).reshape(len(arrays), 2))
    n_out, n_vert = C.c_uint32(0), C.c_uint32(0)
    _check(lib().qm_obstacles_merge(ptrs, sizes, abi.ptr(off, C.c_int32), len(arrays), None, C.byref(n_out), None,
                                    C.byref(n_vert), None))
    outlines = np.zeros(n_out.value, abi.OUTLINE_DTYPE)
    vertices = np.zeros((max(n_vert.value, 1), 2), np.int32)
    envelope = np.zeros(max(n_out.value, 1), np.uint8)
    _check(lib().qm_obstacles_merge(ptrs, sizes, abi.ptr(off, C.c_int32), len(arrays),
                                    outlines.ctypes.data if len(outlines) else None, C.byref(n_out),
                                    abi.ptr(vertices, C.c_int32), C.byref(n_vert), abi.ptr(envelope, C.c_uint8)))
    return outlines, vertices[:n_vert.value], envelope[:n_out.value]


def obstacles_cell_runs(data, column, row, cap=64):
    """The runs of one cell of a tile: [(outline, first edge, edge count), ...]."""
    b, p = _tile_bytes(data)
    runs = np.zeros((cap, 3), np.uint32)
    count = C.c_uint32()
    _check(lib().qm_obstacles_cell_runs(p, len(b), column, row, abi.ptr(runs, C.c_uint32), cap, C.byref(count)))
    return [tuple(int(v) for v in r) for r in runs[:min(count.value, cap)]]


class Skyline:
    """The receiver skyline over a scene's outlines (qm_skyline_build): the index the line
    quadrature's wide buckets query, built on the host."""

    def __init__(self, vertices, outlines, step_m):
        v = np.ascontiguousarray(np.asarray(vertices).reshape(-1, 2), dtype=np.int32)
        o = np.ascontiguousarray(outlines, dtype=abi.OUTLINE_DTYPE)
        handle = C.c_void_p()
        _check(lib().qm_skyline_build(abi.ptr(v, C.c_int32), len(v), o.ctypes.data if len(o) else None, len(o),
                                      float(step_m), C.byref(handle)))
        self.handle = handle

    @classmethod
    def of_scene(cls, scene):
        return cls(scene.vertices, scene.outlines, scene.step_m)

    def close(self):
        if self.handle:
            lib().qm_skyline_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def counts(self):
        cells, runs = C.c_size_t(), C.c_size_t()
        _check(lib().qm_skyline_counts(self.handle, C.byref(cells), C.byref(runs)))
        return cells.value, runs.value

    def arcs(self, receiver_xy, lo_rad, hi_rad, radius_m, floor_m, cap=4096):
        """[n][3] (lo, hi, nearest) for the receiver at scene steps `receiver_xy`."""
        out = np.zeros((cap, 3))
        n = C.c_size_t()
        _check(lib().qm_skyline_arcs(self.handle, int(receiver_xy[0]), int(receiver_xy[1]), float(lo_rad),
                                     float(hi_rad), float(radius_m), float(floor_m), abi.ptr(out, C.c_double), cap,
                                     C.byref(n)))
        return out[:n.value].copy()


def line_quadrature_nodes(start, end, arcs=None, skyline=None, receiver_xy=None, floor_m=0.0,
                          cap=abi.LINE_MAX_NODES):
    """A piece's quadrature nodes (qm_line_quadrature_nodes) and its figures: start and end in
    metres relative to the receiver (x east, y north, z up). The wide buckets see `arcs`
    ([n][3] lo, hi, nearest, handed over whatever the wedge), or the `skyline` index from the
    receiver at scene steps `receiver_xy` above `floor_m`, or nothing."""
    s = np.ascontiguousarray(start, dtype=np.float64)
    e = np.ascontiguousarray(end, dtype=np.float64)
    nodes = np.zeros(cap, dtype=abi.LINE_NODE_DTYPE)
    n = C.c_size_t()
    info = abi.LinePieceInfo()
    query, user = None, None
    keep = []
    if skyline is not None:
        view = abi.SkylineReceiver(skyline.handle, int(receiver_xy[0]), int(receiver_xy[1]), float(floor_m))
        keep.append(view)
        query, user = C.cast(lib().qm_skyline_query, C.c_void_p), C.cast(C.pointer(view), C.c_void_p)
    elif arcs is not None:
        listed = np.asarray(arcs, dtype=np.float64).reshape(-1, 3)

        def hand_over(lo, hi, radius, visit, ctx, _user):
            for a in listed:
                visit(a[0], a[1], a[2], ctx)

        fn = abi.SKYLINE_QUERY_FN(hand_over)
        keep.append(fn)
        query = C.cast(fn, C.c_void_p)
    _check(lib().qm_line_quadrature_nodes(abi.ptr(s, C.c_double), abi.ptr(e, C.c_double), query, user,
                                          nodes.ctypes.data, cap, C.byref(n), C.byref(info)))
    figures = {k: getattr(info, k) for k, _ in abi.LinePieceInfo._fields_}
    return nodes[:n.value].copy(), figures


def distribution_bins(bin_db):
    """The bins of a level-distribution grid of bin_db (qm_distribution_bins)."""
    n = C.c_size_t()
    _check(lib().qm_distribution_bins(float(bin_db), C.byref(n)))
    return n.value


def distribution_with_line(bin_db, bins, silent, values, scale=1.0):
    """A distribution (bins [n][2] of share and share x mean intensity, and its silence) with a
    line of (intensity, share) values times `scale` added (qm_distribution_with_line):
    (bins, silent)."""
    b = np.ascontiguousarray(np.asarray(bins, dtype=np.float64).reshape(-1, 2))
    v = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1, 2))
    out = np.zeros_like(b)
    out_silent = C.c_double()
    _check(lib().qm_distribution_with_line(float(bin_db), abi.ptr(b, C.c_double), float(silent),
                                           abi.ptr(v, C.c_double) if len(v) else None, len(v), float(scale),
                                           abi.ptr(out, C.c_double), C.byref(out_silent)))
    return out, out_silent.value


def distribution_exceeded_db(bin_db, bins, exceeded):
    b = np.ascontiguousarray(np.asarray(bins, dtype=np.float64).reshape(-1, 2))
    level = C.c_double()
    _check(lib().qm_distribution_exceeded_db(float(bin_db), abi.ptr(b, C.c_double), float(exceeded), C.byref(level)))
    return level.value


def distribution_line_values(lam, duty=None, cap=124):
    """A line's (relative intensity, share) values (qm_distribution_line_values): Kurze's quantiles
    at `lam` at the node probabilities, or an event's over its `duty`."""
    out = np.zeros((cap, 2))
    n = C.c_size_t()
    _check(lib().qm_distribution_line_values(float(lam), math.nan if duty is None else float(duty),
                                             abi.ptr(out, C.c_double), cap, C.byref(n)))
    return out[:n.value].copy()


def distribution_pass_values(mean, cap=4096):
    """A stream of passes' (relative intensity, share) values (qm_distribution_pass_values)."""
    out = np.zeros((cap, 2))
    n = C.c_size_t()
    _check(lib().qm_distribution_pass_values(float(mean), abi.ptr(out, C.c_double), cap, C.byref(n)))
    return out[:n.value].copy()


def distribution_layers(bin_db, lines, steady):
    """One period's layers (qm_distribution_layers): `lines` a PERIOD_LINE_DTYPE array, `steady`
    each layer's steady energy. Returns (layer bins [n_layers][n_bins][2], layer silence,
    place bins [n_bins][2], place silence)."""
    rows = np.ascontiguousarray(lines, dtype=abi.PERIOD_LINE_DTYPE)
    st = np.ascontiguousarray(steady, dtype=np.float64)
    n_bins = distribution_bins(bin_db)
    layer_bins = np.zeros((len(st), n_bins, 2))
    layer_silent = np.zeros(len(st))
    place_bins = np.zeros((n_bins, 2))
    place_silent = C.c_double()
    _check(lib().qm_distribution_layers(float(bin_db), rows.ctypes.data if len(rows) else None, len(rows),
                                        abi.ptr(st, C.c_double) if len(st) else None, len(st),
                                        abi.ptr(layer_bins, C.c_double), abi.ptr(layer_silent, C.c_double),
                                        abi.ptr(place_bins, C.c_double), C.byref(place_silent)))
    return layer_bins, layer_silent, place_bins, place_silent.value


def loudness_curve_shape(thirds):
    """A spectrum (28 third-octave energies) at an A-weighted 0 dB, or None without energy."""
    t = np.ascontiguousarray(thirds, dtype=np.float64)
    out = np.zeros(28)
    has = C.c_int()
    _check(lib().qm_loudness_curve_shape(abi.ptr(t, C.c_double), abi.ptr(out, C.c_double), C.byref(has)))
    return out if has.value else None


def distribution_loudness(bin_db, bins, curves):
    """Each period's mean loudness and Nden (qm_distribution_loudness): bins [3][n_bins][2],
    curves [3][191] sone at each whole decibel from -30 dB."""
    b = np.ascontiguousarray(bins, dtype=np.float64)
    c = np.ascontiguousarray(curves, dtype=np.float64)
    mean = np.zeros(3)
    nden = C.c_double()
    _check(lib().qm_distribution_loudness(float(bin_db), abi.ptr(b, C.c_double), abi.ptr(c, C.c_double),
                                          abi.ptr(mean, C.c_double), C.byref(nden)))
    return mean, nden.value


def pixel_read(packed, n_layers, period, cap=4096):
    """One period of a packed pixel (qm_pixel_read): (lines PERIOD_LINE_DTYPE, profiles, steady
    [n_layers], shapes [n_layers + 1][28], has_shape [n_layers + 1])."""
    f = np.ascontiguousarray(packed, dtype=np.float32)
    lines = np.zeros(cap, dtype=abi.PERIOD_LINE_DTYPE)
    profiles = np.zeros(cap, np.int32)
    n = C.c_size_t()
    steady = np.zeros(n_layers)
    shapes = np.zeros((n_layers + 1, 28))
    has = np.zeros(n_layers + 1, np.uint8)
    _check(lib().qm_pixel_read(abi.ptr(f, C.c_float) if len(f) else None, len(f), int(n_layers), int(period),
                               lines.ctypes.data, abi.ptr(profiles, C.c_int32), cap, C.byref(n),
                               abi.ptr(steady, C.c_double), abi.ptr(shapes, C.c_double), abi.ptr(has, C.c_uint8)))
    return lines[:n.value].copy(), profiles[:n.value].copy(), steady, shapes, has.astype(bool)


def distribution_state_means(piece_energy, piece_states, energy):
    """A line's means [3][10] in the weather states from its pieces (qm_distribution_state_means):
    piece_energy [n][3], piece_states [n][2][3] (homogeneous, favourable), energy [3]."""
    pe = np.ascontiguousarray(np.asarray(piece_energy, dtype=np.float64).reshape(-1, 3))
    ps = np.ascontiguousarray(np.asarray(piece_states, dtype=np.float64).reshape(-1, 2, 3))
    en = np.ascontiguousarray(energy, dtype=np.float64)
    out = np.zeros((3, abi.WEATHER_STATES))
    _check(lib().qm_distribution_state_means(abi.ptr(pe, C.c_double) if len(pe) else None,
                                             abi.ptr(ps, C.c_double) if len(ps) else None, len(pe),
                                             abi.ptr(en, C.c_double), abi.ptr(out, C.c_double)))
    return out


def hour_groups(shares, period, runs=0):
    """A period's groups of hours over hourly shares [n_profiles][24] (qm_hour_groups):
    (group_of_slot, group_hours, factors [n_groups][n_profiles])."""
    sh = np.ascontiguousarray(shares, dtype=np.float64).reshape(-1, 24)
    group_of_slot = np.zeros(12, np.uint32)
    group_hours = np.zeros(12, np.uint32)
    factors = np.zeros((12, max(len(sh), 1)))
    n = C.c_size_t()
    _check(lib().qm_hour_groups(abi.ptr(sh, C.c_double) if len(sh) else None, len(sh), int(period), int(runs),
                                abi.ptr(group_of_slot, C.c_uint32), abi.ptr(group_hours, C.c_uint32),
                                abi.ptr(factors, C.c_double), C.byref(n)))
    hours = int(group_hours[:n.value].sum())
    return group_of_slot[:hours].copy(), group_hours[:n.value].copy(), factors[:n.value, :len(sh)].copy()


def pixel_distributions(packed, n_layers, bin_db, shares=None, runs=None):
    """A packed pixel's distributions (qm_pixel_distributions): (layer bins [n_layers][3][n][2],
    layer silence [n_layers][3], place bins [3][n][2], place silence [3])."""
    f = np.ascontiguousarray(packed, dtype=np.float32)
    sh = np.ascontiguousarray(np.zeros((0, 24)) if shares is None else shares, dtype=np.float64).reshape(-1, 24)
    ru = None if runs is None else np.ascontiguousarray(runs, dtype=np.uint32)
    n_bins = distribution_bins(bin_db)
    layer_bins = np.zeros((n_layers, 3, n_bins, 2))
    layer_silent = np.zeros((n_layers, 3))
    place_bins = np.zeros((3, n_bins, 2))
    place_silent = np.zeros(3)
    _check(lib().qm_pixel_distributions(abi.ptr(f, C.c_float) if len(f) else None, len(f), int(n_layers),
                                        float(bin_db), abi.ptr(sh, C.c_double) if len(sh) else None, len(sh),
                                        None if ru is None else abi.ptr(ru, C.c_uint32),
                                        abi.ptr(layer_bins, C.c_double), abi.ptr(layer_silent, C.c_double),
                                        abi.ptr(place_bins, C.c_double), abi.ptr(place_silent, C.c_double)))
    return layer_bins, layer_silent, place_bins, place_silent


def pixel_ndens(packed, n_layers, bin_db, curves, shares=None, runs=None):
    """A packed pixel's Nden per layer and for the place (qm_pixel_ndens): curves
    [n_layers + 1][3][191]."""
    f = np.ascontiguousarray(packed, dtype=np.float32)
    sh = np.ascontiguousarray(np.zeros((0, 24)) if shares is None else shares, dtype=np.float64).reshape(-1, 24)
    ru = None if runs is None else np.ascontiguousarray(runs, dtype=np.uint32)
    cu = np.ascontiguousarray(curves, dtype=np.float64)
    out = np.zeros(n_layers + 1)
    _check(lib().qm_pixel_ndens(abi.ptr(f, C.c_float) if len(f) else None, len(f), int(n_layers), float(bin_db),
                                abi.ptr(sh, C.c_double) if len(sh) else None, len(sh),
                                None if ru is None else abi.ptr(ru, C.c_uint32), abi.ptr(cu, C.c_double),
                                abi.ptr(out, C.c_double)))
    return out


def distribution_percentiles(bin_db, bins):
    """L5, L10, L50 and L90 per period (qm_distribution_percentiles): [4][3] dB from bins [3][n][2]."""
    b = np.ascontiguousarray(bins, dtype=np.float64)
    out = np.zeros((4, 3))
    _check(lib().qm_distribution_percentiles(float(bin_db), abi.ptr(b, C.c_double), abi.ptr(out, C.c_double)))
    return out


def distribution_merge_states(lines, spread):
    """A copy of one period's PERIOD_LINE_DTYPE lines with close weather states merged
    (qm_distribution_merge_states)."""
    rows = np.array(lines, dtype=abi.PERIOD_LINE_DTYPE, copy=True, order="C")
    _check(lib().qm_distribution_merge_states(rows.ctypes.data if len(rows) else None, len(rows), float(spread)))
    return rows


def distribution_layers_grouped(bin_db, lines, steady, hours, group_hours, factors, profiled):
    """One period's layers over groups of hours (qm_distribution_layers_grouped): `factors`
    [n_groups][n_lines] each profiled line's flow in each group against the period's mean."""
    rows = np.ascontiguousarray(lines, dtype=abi.PERIOD_LINE_DTYPE)
    st = np.ascontiguousarray(steady, dtype=np.float64)
    gh = np.ascontiguousarray(group_hours, dtype=np.uint32)
    fa = np.ascontiguousarray(np.asarray(factors, dtype=np.float64).reshape(len(gh), len(rows)))
    pr = np.ascontiguousarray(profiled, dtype=np.uint8)
    n_bins = distribution_bins(bin_db)
    layer_bins = np.zeros((len(st), n_bins, 2))
    layer_silent = np.zeros(len(st))
    place_bins = np.zeros((n_bins, 2))
    place_silent = C.c_double()
    _check(lib().qm_distribution_layers_grouped(
        float(bin_db), rows.ctypes.data if len(rows) else None, len(rows), abi.ptr(st, C.c_double) if len(st) else None,
        len(st), int(hours), abi.ptr(gh, C.c_uint32), len(gh), abi.ptr(fa, C.c_double) if fa.size else None,
        abi.ptr(pr, C.c_uint8) if len(pr) else None, abi.ptr(layer_bins, C.c_double), abi.ptr(layer_silent, C.c_double),
        abi.ptr(place_bins, C.c_double), C.byref(place_silent)))
    return layer_bins, layer_silent, place_bins, place_silent.value


def terrain_decode(data):
    """A terrain tile's window and nodes (qm_terrain_decode): (window dict, height codes uint16
    [rows][columns], impervious, forest and canopy uint8 [rows][columns])."""
    b, p = _tile_bytes(data)
    w = abi.TerrainWindow()
    _check(lib().qm_terrain_decode(p, len(b), C.byref(w), None, None, None, None))
    shape = (w.rows, w.columns)
    heights = np.zeros(shape, np.uint16)
    imp, forest, canopy = (np.zeros(shape, np.uint8) for _ in range(3))
    _check(lib().qm_terrain_decode(p, len(b), C.byref(w), heights.ctypes.data_as(C.POINTER(C.c_uint16)),
                                   abi.ptr(imp, C.c_uint8), abi.ptr(forest, C.c_uint8), abi.ptr(canopy, C.c_uint8)))
    window = dict(north_node=w.north_node, west_node=w.west_node, rows=w.rows, columns=w.columns)
    return window, heights, imp, forest, canopy


def terrain_fine_decode(data):
    """A fine terrain tile's window and details (qm_terrain_fine_decode): (window dict, codes
    int16 [rows][columns], 0.2 m each)."""
    b, p = _tile_bytes(data)
    w = abi.TerrainWindow()
    _check(lib().qm_terrain_fine_decode(p, len(b), C.byref(w), None))
    details = np.zeros((w.rows, w.columns), np.int16)
    _check(lib().qm_terrain_fine_decode(p, len(b), C.byref(w), details.ctypes.data_as(C.POINTER(C.c_int16))))
    return dict(north_node=w.north_node, west_node=w.west_node, rows=w.rows, columns=w.columns), details


def _window(window):
    return abi.TerrainWindow(window["north_node"], window["west_node"], window["rows"], window["columns"])


def mercator_from_degrees(lat, lon):
    """Web Mercator in z12 tile units of a latitude and longitude (qm_mercator_from_degrees)."""
    x, y = C.c_double(), C.c_double()
    lib().qm_mercator_from_degrees(lat, lon, C.byref(x), C.byref(y))
    return x.value, y.value


def terrain_window_of_tile(tile_x, tile_y):
    w = abi.TerrainWindow()
    _check(lib().qm_terrain_window_of_tile(tile_x, tile_y, C.byref(w)))
    return dict(north_node=w.north_node, west_node=w.west_node, rows=w.rows, columns=w.columns)


def terrain_column_of(window, mercator_x):
    w = _window(window)
    return lib().qm_terrain_column_of(C.byref(w), mercator_x)


def terrain_sample(window, heights, impervious, forest, canopy, mercator_xy):
    """The ground at Mercator points over a decoded window (qm_terrain_sample): a list of dicts
    (height_m, ground_factor, forest_cover, canopy_m), None where the reference's sampler refuses."""
    w = _window(window)
    h = np.ascontiguousarray(heights, dtype=np.uint16)
    i, f, c = (np.ascontiguousarray(a, dtype=np.uint8) for a in (impervious, forest, canopy))
    xy = np.ascontiguousarray(np.asarray(mercator_xy, dtype=np.float64).reshape(-1, 2))
    out = (abi.GroundSample * max(len(xy), 1))()
    found = np.zeros(max(len(xy), 1), np.uint8)
    _check(lib().qm_terrain_sample(C.byref(w), h.ctypes.data_as(C.POINTER(C.c_uint16)), abi.ptr(i, C.c_uint8),
                                   abi.ptr(f, C.c_uint8), abi.ptr(c, C.c_uint8), abi.ptr(xy, C.c_double), len(xy),
                                   out, abi.ptr(found, C.c_uint8)))
    return [dict(height_m=out[k].height_m, ground_factor=out[k].ground_factor, forest_cover=out[k].forest_cover,
                 canopy_m=out[k].canopy_m) if found[k] else None for k in range(len(xy))]


def weather_place(table, lat, lon):
    """The weather of a place from the whole weather table's bytes (qm_weather_place):
    (favourable [3][16] in [0, 1], alpha_db_per_km [8])."""
    b, p = _tile_bytes(table)
    fav = np.zeros((abi.PERIODS, abi.SECTORS))
    alpha = np.zeros(abi.BANDS)
    _check(lib().qm_weather_place(p, len(b), lat, lon, abi.ptr(fav, C.c_double), abi.ptr(alpha, C.c_double)))
    return fav, alpha


def weather_read_place(path, lat, lon):
    """The same from the table's file, reading four nodes (qm_weather_read_place)."""
    fav = np.zeros((abi.PERIODS, abi.SECTORS))
    alpha = np.zeros(abi.BANDS)
    _check(lib().qm_weather_read_place(os.fsencode(path), lat, lon, abi.ptr(fav, C.c_double),
                                       abi.ptr(alpha, C.c_double)))
    return fav, alpha


class DeviceScene:
    """A scene uploaded to the device (qm_scene_upload)."""

    def __init__(self, ctx, scene):
        self.ctx = ctx
        self.scene = scene
        self.packed = abi.PackedScene(scene)
        self.handle = C.c_void_p()
        _check(lib().qm_scene_upload(ctx.handle, C.byref(self.packed.desc), C.byref(self.handle)), ctx.handle)

    def close(self):
        if self.handle:
            lib().qm_scene_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def paint_grid(self, grid, histogram=True):
        """The fused painter over `grid`: (bands [cells][8] dB, dBA [cells], Lden [cells],
        histogram [n_bins] or None, stats dict)."""
        g = abi.grid_desc(grid)
        cells = grid.cells
        bands = np.zeros((cells, 8), np.float32)
        dba = np.zeros(cells, np.float32)
        lden = np.zeros(cells, np.float32)
        hist = np.zeros(grid.n_bins, np.uint32) if histogram else None
        stats = abi.PaintStats()
        _check(lib().qm_paint_grid(self.handle, C.byref(g), abi.ptr(bands, C.c_float), abi.ptr(dba, C.c_float),
                                   abi.ptr(lden, C.c_float), abi.ptr(hist, C.c_uint32) if histogram else None,
                                   C.byref(stats)), self.ctx.handle)
        return bands, dba, lden, hist, dict(paths=stats.paths, failed_paths=stats.failed_paths,
                                             crossings=stats.crossings, edge_tests=stats.edge_tests,
                                             vertices=stats.vertices, candidates=stats.candidates,
                                             kernel_ms=stats.kernel_ms, paint_ms=stats.paint_ms)

    def flight_horizons(self, xy_steps, altitude_m, own_footprint, stats=False):
        """Each point's horizons for aircraft screening built on the device (qm_scene_flight_horizons):
        [n][HORIZON_FLOATS] float32, as qm_flight_sums reads them, and the kernel's device time (ms)
        when `stats`."""
        xy = np.ascontiguousarray(np.asarray(xy_steps, dtype=np.float64).reshape(-1, 2))
        alt = np.ascontiguousarray(np.asarray(altitude_m, dtype=np.float64).reshape(-1))
        own = np.ascontiguousarray(np.asarray(own_footprint, dtype=np.uint64).reshape(-1))
        out = np.zeros((len(xy), abi.HORIZON_FLOATS), np.float32)
        ms = C.c_double(0.0)
        _check(lib().qm_scene_flight_horizons(self.handle, abi.ptr(xy, C.c_double), abi.ptr(alt, C.c_double),
                                              abi.ptr(own, C.c_uint64), len(xy), abi.ptr(out, C.c_float),
                                              C.byref(ms)), self.ctx.handle)
        return (out, ms.value) if stats else out

    def surrogate_samples(self, grid):
        """Every path of `grid`: (raw features [rows][32], exact A_boundary labels [rows][8] dB,
        eligible [rows]) with row = cell * n_sources + source offset (terrain scenes: two rows a
        path, homogeneous then favourable)."""
        n_src = (grid.source_end - grid.source_begin) if grid.source_end > grid.source_begin else len(self.scene.sources)
        rows = grid.cells * n_src * (2 if self.scene.dem_altitude is not None else 1)
        g = abi.grid_desc(grid)
        f = np.zeros((rows, 32), np.float32)
        lab = np.zeros((rows, 8), np.float32)
        e = np.zeros(rows, np.uint8)
        _check(lib().qm_surrogate_samples(self.handle, C.byref(g), abi.ptr(f, C.c_float), abi.ptr(lab, C.c_float),
                                          e.ctypes.data_as(C.POINTER(C.c_uint8))), self.ctx.handle)
        return f, lab, e.astype(bool)

    def paint_grid_surrogate(self, grid, net, histogram=True):
        """The painter with the surrogate: like paint_grid, plus stats["surrogate_paths"]."""
        g = abi.grid_desc(grid)
        cells = grid.cells
        bands = np.zeros((cells, 8), np.float32)
        dba = np.zeros(cells, np.float32)
        lden = np.zeros(cells, np.float32)
        hist = np.zeros(grid.n_bins, np.uint32) if histogram else None
        stats = abi.PaintStats()
        taken = C.c_uint64()
        _check(lib().qm_paint_grid_surrogate(self.handle, C.byref(g), net.handle, abi.ptr(bands, C.c_float),
                                             abi.ptr(dba, C.c_float), abi.ptr(lden, C.c_float),
                                             abi.ptr(hist, C.c_uint32) if histogram else None, C.byref(stats),
                                             C.byref(taken)), self.ctx.handle)
        return bands, dba, lden, hist, dict(paths=stats.paths, failed_paths=stats.failed_paths,
                                             crossings=stats.crossings, edge_tests=stats.edge_tests,
                                             vertices=stats.vertices, candidates=stats.candidates,
                                             kernel_ms=stats.kernel_ms, paint_ms=stats.paint_ms,
                                             surrogate_paths=taken.value)

    def evaluate_pairs(self, receiver_xy_m, receiver_height_m, own_footprint, point_of_receiver, source_of_pair,
                       receiver_of_pair, band_weight, n_points, point_bands=None):
        rxy = np.ascontiguousarray(np.asarray(receiver_xy_m, dtype=np.float64).reshape(-1, 2))
        rh = np.ascontiguousarray(receiver_height_m, dtype=np.float32)
        own = np.ascontiguousarray(own_footprint, dtype=np.uint64)
        por = np.ascontiguousarray(point_of_receiver, dtype=np.uint32)
        sop = np.ascontiguousarray(source_of_pair, dtype=np.uint32)
        rop = np.ascontiguousarray(receiver_of_pair, dtype=np.uint32)
        bw = None if band_weight is None else np.ascontiguousarray(band_weight, dtype=np.float32)
        n = len(sop)
        sums = np.zeros((n, abi.PAIR_SUMS), np.float32)
        bands = np.zeros((n, abi.PERIODS, abi.BANDS), np.float32)
        status = np.zeros(n, np.uint32)
        if point_bands is None:
            point_bands = np.zeros((n_points, abi.LAYERS, abi.PERIODS, abi.BANDS), np.float32)
        _check(lib().qm_evaluate_pairs(self.handle, abi.ptr(rxy, C.c_double), abi.ptr(rh, C.c_float),
                                       abi.ptr(own, C.c_uint64), abi.ptr(por, C.c_uint32), len(rxy),
                                       abi.ptr(sop, C.c_uint32), abi.ptr(rop, C.c_uint32),
                                       abi.ptr(bw, C.c_float) if bw is not None else None, n,
                                       abi.ptr(sums, C.c_float), abi.ptr(bands, C.c_float),
                                       abi.ptr(status, C.c_uint32), abi.ptr(point_bands, C.c_float), n_points),
               self.ctx.handle)
        return sums, bands, status, point_bands

    def line_pieces(self, pieces):
        """Sets the scene's line pieces (qm_scene_line_pieces, LINE_SOURCE_DTYPE records): candidate
        n_sources + k of evaluate_pairs is piece k."""
        arr = np.ascontiguousarray(pieces, dtype=abi.LINE_SOURCE_DTYPE)
        _check(lib().qm_scene_line_pieces(self.handle, arr.ctypes.data if len(arr) else None, len(arr)),
               self.ctx.handle)

    def list_crossings(self, frm, to, cap=256):
        frm = np.ascontiguousarray(np.asarray(frm).reshape(-1, 2), dtype=np.int32)
        to = np.ascontiguousarray(np.asarray(to).reshape(-1, 2), dtype=np.int32)
        n = len(frm)
        counts = np.zeros(n, np.uint32)
        status = np.zeros(n, np.uint32)
        edges = np.zeros((n, cap), np.uint32)
        t = np.zeros((n, cap), np.float64)
        flags = np.zeros((n, cap), np.uint32)
        _check(lib().qm_list_crossings(self.handle, abi.ptr(frm, C.c_int32), abi.ptr(to, C.c_int32), n, cap,
                                       abi.ptr(counts, C.c_uint32), abi.ptr(edges, C.c_uint32),
                                       abi.ptr(t, C.c_double), abi.ptr(flags, C.c_uint32),
                                       abi.ptr(status, C.c_uint32)), self.ctx.handle)
        return counts, edges, t, flags, status


def init_params(seed=0):
    """A fresh parameter vector: He-normal weights, zero biases, identity normalisation and
    unbounded ranges (training sets them)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(abi.SURR_PARAMS, np.float32)
    o = 0
    d = abi.SURR_DIMS
    for k in range(5):
        n = d[k + 1] * d[k]
        p[o:o + n] = rng.normal(0.0, np.sqrt(2.0 / d[k]), n).astype(np.float32)
        o += n + d[k + 1]
    q = abi.SURR_WEIGHTS
    p[q + 32:q + 64] = 1.0            # in_scale
    p[q + 72:q + 80] = 1.0            # out_scale
    p[q + 80:q + 112] = -3e38         # feat_lo
    p[q + 112:q + 144] = 3e38         # feat_hi
    p[q + 144:q + 152] = -3e38        # lab_lo
    p[q + 152:q + 160] = 3e38         # lab_hi
    p[q + 160] = 0.0                  # feature set: flat
    return p


class Surrogate:
    """The learned A_boundary network on a device (qm_surrogate_*)."""

    def __init__(self, ctx, params=None, seed=0):
        self.ctx = ctx
        p = np.ascontiguousarray(init_params(seed) if params is None else params, dtype=np.float32)
        if p.shape != (abi.SURR_PARAMS,):
            raise ValueError(f"params must hold {abi.SURR_PARAMS} floats")
        self.handle = C.c_void_p()
        _check(lib().qm_surrogate_create(ctx.handle, abi.ptr(p, C.c_float), C.byref(self.handle)), ctx.handle)

    def close(self):
        if self.handle:
            lib().qm_surrogate_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_kernel(self, kernel):
        """0: the tcgen05 inference kernel (default); 1: the mma.sync one."""
        _check(lib().qm_surrogate_set_kernel(self.handle, kernel), self.ctx.handle)

    def params(self):
        p = np.zeros(abi.SURR_PARAMS, np.float32)
        _check(lib().qm_surrogate_params(self.handle, abi.ptr(p, C.c_float)), self.ctx.handle)
        return p

    def forward(self, features):
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 32)
        out = np.zeros((len(x), 8), np.float32)
        _check(lib().qm_surrogate_forward(self.handle, abi.ptr(x, C.c_float), len(x), abi.ptr(out, C.c_float)),
               self.ctx.handle)
        return out

    def gradients(self, features, labels):
        x = np.ascontiguousarray(features, dtype=np.float32).reshape(-1, 32)
        y = np.ascontiguousarray(labels, dtype=np.float32).reshape(-1, 8)
        g = np.zeros(abi.SURR_WEIGHTS, np.float32)
        loss = C.c_double()
        _check(lib().qm_surrogate_gradients(self.handle, abi.ptr(x, C.c_float), abi.ptr(y, C.c_float), len(x),
                                            abi.ptr(g, C.c_float), C.byref(loss)), self.ctx.handle)
        return g, loss.value

    def train(self, device_scene, grids, epochs=4, batch=16384, learning_rate=2e-3, seed=1, max_samples=0,
              exact_within_m=0.0):
        """Trains on every eligible path of `grids` at least `exact_within_m` long (shorter paths
        stay on the exact path when painting); returns (loss per epoch, samples used)."""
        descs = (abi.GridDesc * len(grids))(*[abi.grid_desc(g) for g in grids])
        cfg = abi.TrainConfig(epochs, batch, learning_rate, seed, max_samples, exact_within_m)
        hist = np.zeros(epochs, np.float64)
        n = C.c_uint64()
        _check(lib().qm_surrogate_train(self.handle, device_scene.handle, descs, len(grids), C.byref(cfg),
                                        abi.ptr(hist, C.c_double), C.byref(n)), self.ctx.handle)
        return hist, n.value


def tile_descs(tiles):
    """ctypes array of qm_tile_desc from dicts (origin, spacing, nx, ny, height_m, source_begin,
    source_end, cell_offset)."""
    arr = (abi.TileDesc * len(tiles))()
    for k, t in enumerate(tiles):
        d = arr[k]
        d.origin[0], d.origin[1] = t["origin"]
        d.spacing, d.nx, d.ny = t["spacing"], t["nx"], t["ny"]
        d.height_m = t.get("height_m", 4.0)
        d.source_begin, d.source_end = t["source_begin"], t["source_end"]
        d.cell_offset = t["cell_offset"]
    return arr


def tile_bucket(tile):
    return lib().qm_tile_bucket(C.byref(tile_descs([tile])[0]))


def tune_default():
    t = abi.TuneTable()
    lib().qm_tune_default(C.byref(t))
    return t


def autotune(device_scene, sample_tiles):
    """(qm_tune_table, timings [buckets][candidates] ms, -1 where not timed)."""
    arr = tile_descs(sample_tiles)
    table = abi.TuneTable()
    timings = np.zeros((abi.TILE_BUCKETS, abi.TILE_CANDIDATES), np.float32)
    _check(lib().qm_batch_autotune(device_scene.handle, arr, len(sample_tiles), C.byref(table),
                                   abi.ptr(timings, C.c_float)), device_scene.ctx.handle)
    return table, timings


class BatchPlan:
    """A planned batch of tiles (qm_batch_plan_*)."""

    def __init__(self, device_scene, tiles, n_cells=None, table=None, graph=True):
        self.dev = device_scene
        arr = tile_descs(tiles)
        self.n_cells = n_cells if n_cells is not None else max(t["cell_offset"] + t["nx"] * t["ny"] for t in tiles)
        self.handle = C.c_void_p()
        _check(lib().qm_batch_plan_create(device_scene.handle, arr, len(tiles), self.n_cells,
                                          C.byref(table) if table is not None else None, 1 if graph else 0,
                                          C.byref(self.handle)), device_scene.ctx.handle)

    def close(self):
        if self.handle:
            lib().qm_batch_plan_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self):
        st = abi.PaintStats()
        _check(lib().qm_batch_plan_run(self.handle, C.byref(st)), self.dev.ctx.handle)
        return dict(paths=st.paths, failed_paths=st.failed_paths, crossings=st.crossings, edge_tests=st.edge_tests,
                    vertices=st.vertices, candidates=st.candidates, kernel_ms=st.kernel_ms, paint_ms=st.paint_ms)

    def read(self):
        bands = np.zeros((self.n_cells, 8), np.float32)
        dba = np.zeros(self.n_cells, np.float32)
        lden = np.zeros(self.n_cells, np.float32)
        _check(lib().qm_batch_plan_read(self.handle, abi.ptr(bands, C.c_float), abi.ptr(dba, C.c_float),
                                        abi.ptr(lden, C.c_float)), self.dev.ctx.handle)
        return bands, dba, lden
