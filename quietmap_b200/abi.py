"""ctypes mirror of include/qm_batch.h: the structs and constants of the C ABI.

A Rust painter binds the same structs through its own FFI declarations; this module is the Python
binding used by the host mirror of `paint::exact::Batch`, the tests and the benchmark.
"""

import ctypes as C

import numpy as np

ABI_VERSION = 3
BANDS = 8
PERIODS = 3
SECTORS = 16
LAYERS = 6
THIRDS = 28
CELL_NO_LEVEL, CELL_SILENCE = 255, 254
HM3_TILE_PX = 512
HM3_STREAM_BYTES = 6 + HM3_TILE_PX * HM3_TILE_PX
PAIR_SUMS = 9
POINT_BANDS = LAYERS * PERIODS * BANDS

QM_OK = 0
QM_ERR_ARGUMENT = 1
QM_ERR_CUDA = 2
QM_ERR_CAPACITY = 3
QM_ERR_TIMEOUT = 4
QM_ERR_UNSUPPORTED = 5

FAILED_NOT_READ = 1
FAILED_NO_TERRAIN = 2
FAILED_CAPACITY = 4
FAILED_LINE_CUTOFF = 8
FAILED_TIMEOUT = 16


class TerrainWindow(C.Structure):
    _fields_ = [("north_node", C.c_int32), ("west_node", C.c_int32), ("rows", C.c_uint32), ("columns", C.c_uint32)]


class GroundSample(C.Structure):
    _fields_ = [("height_m", C.c_double), ("ground_factor", C.c_double), ("forest_cover", C.c_double),
                ("canopy_m", C.c_double)]


class ObstaclesCounts(C.Structure):
    _fields_ = [(name, C.c_uint32) for name in
                ("outlines", "vertices", "runs", "occupied_cells", "footprint_squares", "pad_")]


class Outline(C.Structure):
    _fields_ = [
        ("first_vertex", C.c_uint32),
        ("vertex_count", C.c_uint32),
        ("footprint_id", C.c_uint64),
        ("height_m", C.c_float),
        ("building", C.c_uint32),
    ]


class Source(C.Structure):
    _fields_ = [
        ("x", C.c_int32),
        ("y", C.c_int32),
        ("height_m", C.c_float),
        ("ground_factor", C.c_float),
        ("exclusion_radius_m", C.c_float),
        ("platform_half_width_m", C.c_float),
        ("footprint_id", C.c_uint64),
        ("layer", C.c_uint32),
        ("pad_", C.c_uint32),
        ("energy", (C.c_float * BANDS) * PERIODS),
    ]


class SceneDesc(C.Structure):
    _fields_ = [
        ("step_m", C.c_double),
        ("cell_steps", C.c_int32),
        ("extent_steps", C.c_int32 * 2),
        ("n_vertices", C.c_uint32),
        ("vertices", C.POINTER(C.c_int32)),
        ("n_outlines", C.c_uint32),
        ("outlines", C.POINTER(Outline)),
        ("dem_nx", C.c_int32),
        ("dem_ny", C.c_int32),
        ("dem_origin", C.c_int32 * 2),
        ("dem_spacing", C.c_int32),
        ("dem_altitude_m", C.POINTER(C.c_float)),
        ("dem_ground_factor", C.POINTER(C.c_float)),
        ("flat_altitude_m", C.c_float),
        ("flat_ground_factor", C.c_float),
        ("n_sources", C.c_uint32),
        ("sources", C.POINTER(Source)),
        ("favourable", (C.c_float * SECTORS) * PERIODS),
        ("alpha_db_per_km", C.c_float * BANDS),
    ]


class GridDesc(C.Structure):
    _fields_ = [
        ("origin", C.c_int32 * 2),
        ("spacing", C.c_int32),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("height_m", C.c_float),
        ("source_begin", C.c_uint32),
        ("source_end", C.c_uint32),
        ("level_min_db", C.c_double),
        ("bin_db", C.c_double),
        ("n_bins", C.c_uint32),
    ]


class PaintStats(C.Structure):
    _fields_ = [
        ("paths", C.c_uint64),
        ("failed_paths", C.c_uint64),
        ("crossings", C.c_uint64),
        ("edge_tests", C.c_uint64),
        ("vertices", C.c_uint64),
        ("candidates", C.c_uint64),
        ("kernel_ms", C.c_double),
        ("paint_ms", C.c_double),
    ]


# numpy structured dtypes with the same layout (one upload of many records at once).
OUTLINE_DTYPE = np.dtype(
    [("first_vertex", "<u4"), ("vertex_count", "<u4"), ("footprint_id", "<u8"),
     ("height_m", "<f4"), ("building", "<u4")], align=True)
SOURCE_DTYPE = np.dtype(
    [("x", "<i4"), ("y", "<i4"), ("height_m", "<f4"), ("ground_factor", "<f4"),
     ("exclusion_radius_m", "<f4"), ("platform_half_width_m", "<f4"), ("footprint_id", "<u8"),
     ("layer", "<u4"), ("pad_", "<u4"), ("energy", "<f4", (PERIODS, BANDS))], align=True)
# qm_line_source: a line piece candidate's ends (steps) and its source properties (energy per metre).
LINE_SOURCE_DTYPE = np.dtype([("a", "<f8", (2,)), ("b", "<f8", (2,)), ("source", SOURCE_DTYPE)], align=True)

AIRCRAFT_TYPE_DTYPE = np.dtype(
    [("sel_db", "<f4", (2, 10, 10)), ("lamax_db", "<f4", (2, 10, 10)), ("v_ref_kt", "<f4"), ("installation", "<u4"),
     ("spectrum_db", "<f4", (THIRDS,)), ("pad_", "<u4", (2,))], align=True)
FLIGHT_SEGMENT_DTYPE = np.dtype(
    [("start", "<f4", (3,)), ("end", "<f4", (3,)), ("power", "<f4"), ("speed_mps", "<f4"), ("type", "<u4"),
     ("departure", "<u4"), ("flight", "<u4"), ("pad_", "<u4")], align=True)

# include/qm_flights.h: a square's aircraft boxes, lattice points and their segments of boxes.
PASS_CLASSES = 48
FLIGHT_SUMS = PERIODS + 2 * PERIODS * PASS_CLASSES
TERRAIN_SECTORS, BUILDING_SECTORS, HORIZON_BANDS = 32, 256, 6
TERRAIN_HORIZON_FLOATS = 1 + TERRAIN_SECTORS * (1 + 2 * HORIZON_BANDS)
HORIZON_FLOATS = TERRAIN_HORIZON_FLOATS + 1 + BUILDING_SECTORS * (1 + 2 * HORIZON_BANDS)
FLIGHT_WEIGHT_ONE, FLIGHT_WEIGHT_FAR, FLIGHT_WEIGHT_NEAR = 0, 1, 2
FLIGHT_BOX_DTYPE = np.dtype(
    [("east_m", "<f8"), ("north_m", "<f8"), ("centroid_altitude_m", "<f8"), ("ground_m", "<f8"), ("axis_rad", "<f8"),
     ("gradient", "<f8"), ("gradient_spread", "<f8"), ("piece_length_m", "<f8", (PERIODS,)),
     ("levels_db", "<f8", (PERIODS, 10)), ("tail_levels_db", "<f8", (PERIODS,)), ("lg_scaled_distance", "<f8", (10,)),
     ("installation_shares", "<f8", (PERIODS, 2, 3)), ("passing", "<f8", (PERIODS,)), ("helicopter", "<u4"),
     ("pad_", "<u4")], align=True)
FLIGHT_POINT_DTYPE = np.dtype(
    [("x", "<f8"), ("y", "<f8"), ("altitude_m", "<f8"), ("horizons", "<u8"), ("impedance_gain", "<f8")], align=True)
BOX_SEGMENT_DTYPE = np.dtype(
    [("within_m", "<f8"), ("coarse_m", "<f8"), ("point", "<u4"), ("sum", "<u4"), ("first", "<u4"), ("count", "<u4"),
     ("weight", "<u4"), ("pad_", "<u4")], align=True)
assert FLIGHT_BOX_DTYPE.itemsize == 600 and FLIGHT_POINT_DTYPE.itemsize == 40 and BOX_SEGMENT_DTYPE.itemsize == 40


class FlightSumsStats(C.Structure):
    _fields_ = [("box_reads", C.c_uint64), ("boxes_heard", C.c_uint64), ("kernel_ms", C.c_double)]


LINE_NODE_DTYPE = np.dtype([("along_m", "<f8"), ("weight_rad", "<f8"), ("obstacles_on_ray", "<u4"),
                            ("reserved", "<u4")], align=True)
LINE_MAX_NODES = 705
DISTRIBUTION_MAX_BINS = 1800
DISTRIBUTION_LINE_NODES = 124
WEATHER_STATES = 10
PERIOD_LINE_DTYPE = np.dtype([("layer", "<u4"), ("reserved", "<u4"), ("energy", "<f8"),
                              ("means", "<f8", (WEATHER_STATES,)), ("lambda", "<f8"), ("duty", "<f8"),
                              ("passing", "<f8")], align=True)


class LinePieceInfo(C.Structure):
    _fields_ = [("length_m", C.c_double), ("subtended_angle_rad", C.c_double), ("divergence_factor", C.c_double),
                ("start_angle_rad", C.c_double)]


class SkylineReceiver(C.Structure):
    _fields_ = [("skyline", C.c_void_p), ("x", C.c_int64), ("y", C.c_int64), ("floor_m", C.c_double)]


# A skyline query's visit and the query itself (qm_skyline_visit_fn, qm_skyline_query_fn).
SKYLINE_VISIT_FN = C.CFUNCTYPE(None, C.c_double, C.c_double, C.c_double, C.c_void_p)
SKYLINE_QUERY_FN = C.CFUNCTYPE(None, C.c_double, C.c_double, C.c_double, SKYLINE_VISIT_FN, C.c_void_p, C.c_void_p)


class FlightGridDesc(C.Structure):
    _fields_ = [
        ("origin_m", C.c_double * 2),
        ("spacing_m", C.c_double),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("receiver_height_m", C.c_float),
        ("pad_", C.c_float),
        ("reach_m", C.c_double),
        ("duration_s", C.c_double),
    ]


class FlightStats(C.Structure):
    _fields_ = [("pairs", C.c_uint64), ("pairs_in_reach", C.c_uint64), ("kernel_ms", C.c_double),
                ("loudness_ms", C.c_double)]


def flight_grid_desc(grid):
    g = FlightGridDesc()
    g.origin_m[0], g.origin_m[1] = grid["origin_m"]
    g.spacing_m = grid["spacing_m"]
    g.nx, g.ny = grid["nx"], grid["ny"]
    g.receiver_height_m = grid["receiver_height_m"]
    g.reach_m = grid["reach_m"]
    g.duration_s = grid["duration_s"]
    return g


assert AIRCRAFT_TYPE_DTYPE.itemsize == 4 * (200 + 200 + 2 + 28 + 2)
assert FLIGHT_SEGMENT_DTYPE.itemsize == 48
assert OUTLINE_DTYPE.itemsize == C.sizeof(Outline)
assert SOURCE_DTYPE.itemsize == C.sizeof(Source)
assert LINE_NODE_DTYPE.itemsize == 24
assert PERIOD_LINE_DTYPE.itemsize == 120


def ptr(array, ctype):
    """A ctypes pointer into a contiguous numpy array (None for None)."""
    if array is None:
        return None
    if not array.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return array.ctypes.data_as(C.POINTER(ctype))


class PackedScene:
    """A scene descriptor with the numpy arrays it points into kept alive."""

    def __init__(self, scene):
        self.scene = scene
        self.vertices = np.ascontiguousarray(scene.vertices, dtype=np.int32).reshape(-1, 2)
        self.outlines = np.ascontiguousarray(scene.outlines, dtype=OUTLINE_DTYPE)
        self.sources = np.ascontiguousarray(scene.sources, dtype=SOURCE_DTYPE)
        d = SceneDesc()
        d.step_m = scene.step_m
        d.cell_steps = scene.cell_steps
        d.extent_steps[0], d.extent_steps[1] = scene.extent_steps
        d.n_vertices = len(self.vertices)
        d.vertices = ptr(self.vertices, C.c_int32)
        d.n_outlines = len(self.outlines)
        d.outlines = self.outlines.ctypes.data_as(C.POINTER(Outline))
        if scene.dem_altitude is not None:
            self.dem_z = np.ascontiguousarray(scene.dem_altitude, dtype=np.float32)
            self.dem_g = np.ascontiguousarray(scene.dem_ground_factor, dtype=np.float32)
            d.dem_ny, d.dem_nx = self.dem_z.shape
            d.dem_origin[0], d.dem_origin[1] = scene.dem_origin
            d.dem_spacing = scene.dem_spacing
            d.dem_altitude_m = ptr(self.dem_z, C.c_float)
            d.dem_ground_factor = ptr(self.dem_g, C.c_float)
        else:
            d.dem_nx = d.dem_ny = 0
        d.flat_altitude_m = scene.flat_altitude_m
        d.flat_ground_factor = scene.flat_ground_factor
        d.n_sources = len(self.sources)
        d.sources = self.sources.ctypes.data_as(C.POINTER(Source))
        fav = np.asarray(scene.favourable, dtype=np.float32).reshape(PERIODS, SECTORS)
        for p in range(PERIODS):
            for s in range(SECTORS):
                d.favourable[p][s] = float(fav[p, s])
        for b in range(BANDS):
            d.alpha_db_per_km[b] = float(scene.alpha_db_per_km[b])
        self.desc = d


SURR_FEATURES, SURR_HIDDEN, SURR_OUTPUTS = 32, 256, 8
SURR_DIMS = (32, 256, 256, 256, 256, 8)
SURR_WEIGHTS = sum(SURR_DIMS[k + 1] * SURR_DIMS[k] + SURR_DIMS[k + 1] for k in range(5))
SURR_PARAMS = SURR_WEIGHTS + 32 + 32 + 8 + 8 + 32 + 32 + 8 + 8 + 1


class TrainConfig(C.Structure):
    _fields_ = [
        ("epochs", C.c_uint32),
        ("batch", C.c_uint32),
        ("learning_rate", C.c_float),
        ("seed", C.c_uint32),
        ("max_samples", C.c_uint32),
        ("exact_within_m", C.c_float),
    ]


class TileDesc(C.Structure):
    _fields_ = [
        ("origin", C.c_int32 * 2),
        ("spacing", C.c_int32),
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("height_m", C.c_float),
        ("source_begin", C.c_uint32),
        ("source_end", C.c_uint32),
        ("cell_offset", C.c_uint64),
    ]


class TileConfig(C.Structure):
    _fields_ = [("block_w", C.c_uint32), ("block_h", C.c_uint32), ("threads", C.c_uint32), ("chunk", C.c_uint32)]


TILE_BUCKETS, TILE_CANDIDATES = 4, 25


class TuneTable(C.Structure):
    _fields_ = [("bucket", TileConfig * TILE_BUCKETS)]


def grid_desc(grid):
    g = GridDesc()
    g.origin[0], g.origin[1] = grid.origin
    g.spacing = grid.spacing
    g.nx, g.ny = grid.nx, grid.ny
    g.height_m = grid.height_m
    g.source_begin, g.source_end = grid.source_begin, grid.source_end
    g.level_min_db = grid.level_min_db
    g.bin_db = grid.bin_db
    g.n_bins = grid.n_bins
    return g
