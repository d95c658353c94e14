"""ctypes wrapper of the FP64 CPU oracle (oracle/libqm_oracle.so) — TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's CPU physics (quietmap's Rust `physics`, `popup` and `paint`
crates) in C++ double precision; each C function cites the reference file:line it follows.
Only tests/, the smoke check and the benchmark's CPU-baseline leg import this module; the
product path (quietmap_b200) never does.
"""

import ctypes as C
import os
import subprocess

import numpy as np

from quietmap_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqm_oracle.so")

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_U64 = C.POINTER(C.c_uint64)
_U32 = C.POINTER(C.c_uint32)
_I32 = C.POINTER(C.c_int32)


def build():
    """Compiles the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.qmo_alpha_bands.argtypes = [C.c_double, C.c_double, _D]
        L.qmo_state_boundaries.argtypes = [_D, _D, _D, C.c_size_t, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_double, _D, C.c_size_t, _D, C.c_size_t, _D, _D]
        L.qmo_ray_terms.argtypes = [
            C.c_double, _D, _D, _D, C.c_size_t, _D, _D, _I32, _I32, _U64, C.c_size_t,
            C.c_double, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double, C.c_uint64,
            _D, _D, _D, _D, _D, _D, _D, _D, C.c_size_t, C.POINTER(C.c_size_t), _D, C.c_size_t,
            C.POINTER(C.c_size_t)]
        L.qmo_crests_of.argtypes = [_D, C.c_size_t, C.c_double, _D, C.c_size_t]
        L.qmo_crests_of.restype = C.c_size_t
        L.qmo_scene_new.argtypes = [C.POINTER(abi.SceneDesc)]
        L.qmo_scene_new.restype = C.c_void_p
        L.qmo_scene_free.argtypes = [C.c_void_p]
        L.qmo_crossings.argtypes = [C.c_void_p, _I64, _I64, _D, _U64, _U32, _I32, _I32, C.c_size_t]
        L.qmo_crossings.restype = C.c_size_t
        L.qmo_enclosing_buildings.argtypes = [C.c_void_p, _I64, C.c_size_t, _U64, C.c_int]
        L.qmo_profile.argtypes = [C.c_void_p, _I64, _I64, _D, _D, _D, C.c_size_t, _D]
        L.qmo_profile.restype = C.c_size_t
        L.qmo_evaluate_pairs.argtypes = [C.c_void_p, _I64, _D, _U64, _U32, C.c_size_t, _U32, _U32, _D,
                                         C.c_size_t, _D, _D, _D, C.c_size_t, C.c_int]
        L.qmo_path_counts.argtypes = [C.c_void_p, _I64, _I64, _D]
        L.qmo_path_counts.restype = None
        L.qmo_paint_grid.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), C.c_uint32, C.c_uint32, _D, _D,
                                     C.c_int, _U64]
        L.qmo_zwicker.argtypes = [_D]
        L.qmo_zwicker.restype = C.c_double
        L.qmo_zwicker_many.argtypes = [_D, C.c_size_t, _D, C.c_int]
        L.qmo_level_histogram.argtypes = [_D, C.c_size_t, C.c_double, C.c_double, C.c_uint32, _U32]
        L.qmo_level_bin.argtypes = [C.c_double, C.c_double, C.c_double, C.c_uint32]
        L.qmo_level_bin.restype = C.c_uint32
        _B = C.POINTER(C.c_uint8)
        L.qmo_percentile_table.argtypes = [C.c_int, C.POINTER(C.c_float)]
        L.qmo_percentile_table.restype = None
        L.qmo_relative_intensities.argtypes = [C.c_double, _D, C.c_size_t, _D]
        L.qmo_relative_intensities.restype = None
        L.qmo_ground_attenuation_bands.argtypes = [C.c_double] * 9 + [C.c_int, _D]
        L.qmo_ground_attenuation_bands.restype = None
        for name in ("qmo_crossings_d", "qmo_crossings_every"):
            f = getattr(L, name)
            f.argtypes = [C.c_void_p, _D, _D, _D, _U64, _U32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_size_t]
            f.restype = C.c_size_t
        L.qmo_profile_d.argtypes = [C.c_void_p, _D, _D, _D, _D, _D, C.c_size_t, _D]
        L.qmo_profile_d.restype = C.c_size_t
        L.qmo_line_piece.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.c_double, C.c_uint64, _D, _D, C.c_void_p,
                                     C.c_int, _D, C.c_size_t, _D, _D]
        L.qmo_line_piece.restype = C.c_int
        L.qmo_skyline_arcs.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.c_double, C.c_double, C.c_double,
                                       C.c_double, _D, C.c_size_t]
        L.qmo_skyline_arcs.restype = C.c_size_t
        L.qmo_scene_line_nodes.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.c_double, _D, _D, _D, _D,
                                           C.POINTER(C.c_uint8), C.c_size_t]
        L.qmo_scene_line_nodes.restype = C.c_int
        L.qmo_path_difference.argtypes = [C.c_int, C.c_double, _D, _D, _D, _D, C.c_size_t, _D]
        L.qmo_path_difference.restype = C.c_double
        L.qmo_diffraction_path.argtypes = [C.c_int, C.c_double, _D, _D, _D, C.c_size_t, _D,
                                           C.POINTER(C.c_size_t), _D, C.POINTER(C.c_size_t), C.c_size_t]
        L.qmo_diffraction_path.restype = C.c_int
        L.qmo_state_ray_altitude.argtypes = [C.c_int, C.c_double, _D, _D, _D, _D, C.c_double]
        L.qmo_state_ray_altitude.restype = C.c_double
        L.qmo_line_geometry.argtypes = [_D, _D, _D]
        L.qmo_line_geometry.restype = C.c_int
        L.qmo_line_in_plane_angle_at.argtypes = [_D, _D, C.c_double]
        L.qmo_line_in_plane_angle_at.restype = C.c_double
        L.qmo_line_nodes.argtypes = [_D, _D, _D, C.c_size_t, _D, _D, _B, C.c_size_t]
        L.qmo_line_nodes.restype = C.c_int
        L.qmo_favourable_at.argtypes = [C.POINTER(C.c_float), C.c_double]
        L.qmo_favourable_at.restype = C.c_double
        L.qmo_nden_cell.argtypes = [C.c_double]
        L.qmo_nden_cell.restype = C.c_uint8
        L.qmo_lden_cell.argtypes = [C.c_double]
        L.qmo_lden_cell.restype = C.c_int
        L.qmo_quantize_cells.argtypes = [_D, _D, _B, C.c_size_t, _B, _B]
        L.qmo_quantize_cells.restype = C.c_int64
        L.qmo_hm3_predict.argtypes = [_B, C.c_uint8, C.c_int, _B]
        L.qmo_hm3_predict.restype = C.c_int
        L.qmo_hm3_unpredict.argtypes = [_B]
        L.qmo_hm3_unpredict.restype = None
        for name in ("qmo_lateral_attenuation_db", "qmo_speed_correction_db"):
            getattr(L, name).argtypes = [C.c_double, C.c_double]
            getattr(L, name).restype = C.c_double
        L.qmo_finite_segment_energy_fraction.argtypes = [C.c_double, C.c_double, C.c_double]
        L.qmo_finite_segment_energy_fraction.restype = C.c_double
        L.qmo_installation_energy_gain.argtypes = [C.c_uint32, C.c_double, C.c_double]
        L.qmo_installation_energy_gain.restype = C.c_double
        L.qmo_npd_level.argtypes = [_D, C.c_double, C.c_double]
        L.qmo_npd_level.restype = C.c_double
        L.qmo_tail_absorption.argtypes = [_D]
        L.qmo_tail_absorption.restype = C.c_double
        L.qmo_surrogate_samples.argtypes = [C.c_void_p, C.POINTER(abi.GridDesc), C.c_uint32, C.c_uint32, _D, _D,
                                            C.POINTER(C.c_uint8), C.c_int]
        L.qmo_flight_grid.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_size_t, C.POINTER(abi.FlightGridDesc),
                                      C.c_uint32, C.c_uint32, _D, _D, _D, C.c_int]
        for name in ("qmo_path_difference_loss_db",):
            getattr(L, name).argtypes = [C.c_double]
            getattr(L, name).restype = C.c_double
        for name in ("qmo_edge_loss_db", "qmo_screened_sel_db"):
            getattr(L, name).argtypes = [C.c_double] * 4
            getattr(L, name).restype = C.c_double
        L.qmo_flight_horizons.argtypes = [C.c_void_p, _D, _D, _U64, C.c_size_t, C.POINTER(C.c_float), C.c_int]
        L.qmo_flight_horizons.restype = None
        L.qmo_flight_weight.argtypes = [C.c_uint32, C.c_double, C.c_double]
        L.qmo_flight_weight.restype = C.c_double
        L.qmo_horizon_loss_db.argtypes = [C.POINTER(C.c_float), C.c_int, _D]
        L.qmo_horizon_loss_db.restype = C.c_double
        L.qmo_segment_sel_db.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double]
        L.qmo_segment_sel_db.restype = C.c_double
        L.qmo_box_sums.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, _D, C.c_void_p]
        L.qmo_box_sums.restype = C.c_int
        L.qmo_box_sel.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), _D, _D]
        L.qmo_box_sel.restype = None
        L.qmo_flight_sums.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_float), C.c_void_p, C.c_size_t, _D,
                                      C.c_size_t, C.c_int]
        L.qmo_flight_sums.restype = C.c_uint64
        _lib = L
    return _lib


def threads():
    return max(os.cpu_count() or 1, 1)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def alpha_bands(temperature_c, rh):
    out = np.zeros(8)
    lib().qmo_alpha_bands(temperature_c, rh, abi.ptr(out, C.c_double))
    return out


def state_boundaries(d, z, g, source, receiver, source_gf, terrain, tops):
    """A_boundary of both states of a vertical path: ([2][8] attenuation, [2][8] no-ground)."""
    d, z, g = _d(d), _d(z), _d(g)
    terrain = _d(np.asarray(terrain, dtype=np.float64).reshape(-1, 2))
    tops = _d(np.asarray(tops, dtype=np.float64).reshape(-1, 2))
    att = np.zeros(16)
    wog = np.zeros(16)
    lib().qmo_state_boundaries(abi.ptr(d, C.c_double), abi.ptr(z, C.c_double), abi.ptr(g, C.c_double), len(d),
                               source[0], source[1], receiver[0], receiver[1], source_gf,
                               abi.ptr(terrain, C.c_double), len(terrain), abi.ptr(tops, C.c_double), len(tops),
                               abi.ptr(att, C.c_double), abi.ptr(wog, C.c_double))
    return att.reshape(2, 8), wog.reshape(2, 8)


def ray_terms(horizontal_m, t, ground_m, ground_factor, crossings, ends, p, alpha):
    """One ray's transfer; crossings rows (t, height, building, bounds_roof, footprint)."""
    t, zg, gf = _d(t), _d(ground_m), _d(ground_factor)
    ct = _d([c[0] for c in crossings])
    ch = _d([c[1] for c in crossings])
    cb = np.ascontiguousarray([int(c[2]) for c in crossings], dtype=np.int32)
    cr = np.ascontiguousarray([int(c[3]) for c in crossings], dtype=np.int32)
    cf = np.ascontiguousarray([c[4] for c in crossings], dtype=np.uint64)
    p, alpha = _d(p), _d(alpha)
    slant = np.zeros(1)
    periods = np.zeros(24)
    states = np.zeros(16)
    cap = 4096
    pd, pz, pg = np.zeros(cap), np.zeros(cap), np.zeros(cap)
    tops = np.zeros(2 * cap)
    n_path = C.c_size_t()
    n_tops = C.c_size_t()
    sg = ends.get("source_ground_m")
    sgf = ends.get("source_ground_factor")
    lib().qmo_ray_terms(horizontal_m, abi.ptr(t, C.c_double), abi.ptr(zg, C.c_double), abi.ptr(gf, C.c_double),
                        len(t), abi.ptr(ct, C.c_double), abi.ptr(ch, C.c_double), abi.ptr(cb, C.c_int32),
                        abi.ptr(cr, C.c_int32), abi.ptr(cf, C.c_uint64), len(ct), ends["source_height_m"],
                        int(sg is not None), float(sg or 0.0), ends["receiver_altitude_m"],
                        int(sgf is not None), float(sgf or 0.0), ends.get("platform_half_width_m", 0.0),
                        ends.get("own_footprint", 0), abi.ptr(p, C.c_double), abi.ptr(alpha, C.c_double),
                        abi.ptr(slant, C.c_double), abi.ptr(periods, C.c_double), abi.ptr(states, C.c_double),
                        abi.ptr(pd, C.c_double), abi.ptr(pz, C.c_double), abi.ptr(pg, C.c_double), cap,
                        C.byref(n_path), abi.ptr(tops, C.c_double), cap, C.byref(n_tops))
    n, m = n_path.value, n_tops.value
    return dict(slant_m=slant[0], periods=periods.reshape(3, 8), states=states.reshape(2, 8),
                path_d=pd[:n].copy(), path_z=pz[:n].copy(), path_g=pg[:n].copy(),
                tops=tops[:2 * m].reshape(m, 2).copy())


def crests_of(points, length):
    xz = _d(np.asarray(points, dtype=np.float64).reshape(-1, 2))
    out = np.zeros(2 * max(len(xz), 1))
    n = lib().qmo_crests_of(abi.ptr(xz, C.c_double), len(xz), length, abi.ptr(out, C.c_double), len(xz))
    return out[:2 * n].reshape(n, 2)


class OracleScene:
    """The oracle's copy of a scene (its own cell lists), built from the ABI descriptor."""

    def __init__(self, scene):
        self.packed = abi.PackedScene(scene)
        self.scene = scene
        self.handle = lib().qmo_scene_new(C.byref(self.packed.desc))

    def __del__(self):
        if getattr(self, "handle", None):
            lib().qmo_scene_free(self.handle)
            self.handle = None

    def crossings(self, frm, to, cap=4096):
        frm = np.ascontiguousarray(frm, dtype=np.int64)
        to = np.ascontiguousarray(to, dtype=np.int64)
        t = np.zeros(cap)
        fp = np.zeros(cap, np.uint64)
        edge = np.zeros(cap, np.uint32)
        br = np.zeros(cap, np.int32)
        bd = np.zeros(cap, np.int32)
        n = lib().qmo_crossings(self.handle, abi.ptr(frm, C.c_int64), abi.ptr(to, C.c_int64),
                                abi.ptr(t, C.c_double), abi.ptr(fp, C.c_uint64), abi.ptr(edge, C.c_uint32),
                                abi.ptr(br, C.c_int32), abi.ptr(bd, C.c_int32), cap)
        n = min(n, cap)
        return dict(t=t[:n].copy(), footprint=fp[:n].copy(), edge=edge[:n].copy(),
                    bounds_roof=br[:n].astype(bool), building=bd[:n].astype(bool))

    def _crossings_f64(self, fn, frm, to, cap=4096):
        frm = np.ascontiguousarray(frm, dtype=np.float64)
        to = np.ascontiguousarray(to, dtype=np.float64)
        t = np.zeros(cap)
        fp = np.zeros(cap, np.uint64)
        edge = np.zeros(cap, np.uint32)
        br = np.zeros(cap, np.int32)
        bd = np.zeros(cap, np.int32)
        n = fn(self.handle, abi.ptr(frm, C.c_double), abi.ptr(to, C.c_double), abi.ptr(t, C.c_double),
               abi.ptr(fp, C.c_uint64), abi.ptr(edge, C.c_uint32), abi.ptr(br, C.c_int32), abi.ptr(bd, C.c_int32),
               cap)
        n = min(n, cap)
        return dict(t=t[:n].copy(), footprint=fp[:n].copy(), edge=edge[:n].copy(),
                    bounds_roof=br[:n].astype(bool), building=bd[:n].astype(bool))

    def crossings_f64(self, frm, to):
        """The walk's crossing list for ends anywhere (f64 steps)."""
        return self._crossings_f64(lib().qmo_crossings_d, frm, to)

    def flight_horizons(self, xy_steps, altitude_m, own_footprint, nthreads=None):
        """Each point's horizons for aircraft screening (Horizons::build), [n][HORIZON_FLOATS]
        float32 as the card keeps them."""
        xy = np.ascontiguousarray(np.asarray(xy_steps, dtype=np.float64).reshape(-1, 2))
        alt = np.ascontiguousarray(np.asarray(altitude_m, dtype=np.float64).reshape(-1))
        own = np.ascontiguousarray(np.asarray(own_footprint, dtype=np.uint64).reshape(-1))
        out = np.zeros((len(xy), abi.HORIZON_FLOATS), np.float32)
        lib().qmo_flight_horizons(self.handle, abi.ptr(xy, C.c_double), abi.ptr(alt, C.c_double),
                                  abi.ptr(own, C.c_uint64), len(xy), abi.ptr(out, C.c_float), nthreads or threads())
        return out

    def crossings_every(self, frm, to):
        """Every edge against the ray with the walk's deduplication: the list the walk must give."""
        return self._crossings_f64(lib().qmo_crossings_every, frm, to)

    def profile_f64(self, frm, to, cap=65536):
        """The ground profile under a ray with ends anywhere: (horizontal metres, t, altitude, G), as
        `profile` gives it."""
        frm = np.ascontiguousarray(frm, dtype=np.float64)
        to = np.ascontiguousarray(to, dtype=np.float64)
        t, z, g = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        h = np.zeros(1)
        n = lib().qmo_profile_d(self.handle, abi.ptr(frm, C.c_double), abi.ptr(to, C.c_double), abi.ptr(t, C.c_double),
                                abi.ptr(z, C.c_double), abi.ptr(g, C.c_double), cap, abi.ptr(h, C.c_double))
        n = min(n, cap)
        return float(h[0]), t[:n].copy(), z[:n].copy(), g[:n].copy()

    def line_piece(self, receiver_xy, receiver_altitude_m, a, b, source, arcs=None, own_footprint=0):
        """A line piece's received energy at a lattice receiver (physics/src/line.rs quadrature,
        popup/src/evaluate.rs:215-265): (bands [3][8], states [2][3], quadrature nodes). `a`, `b`
        are the piece's ends in steps (anywhere); `source` a SOURCE_DTYPE record whose energy is
        the power per metre. The quadrature sees the scene's skyline from the receiver, or with
        `arcs` ([n][3] azimuth lo, hi, nearest) those arcs whatever the wedge."""
        rxy = np.ascontiguousarray(receiver_xy, dtype=np.int64)
        pa, pb = np.ascontiguousarray(a, dtype=np.float64), np.ascontiguousarray(b, dtype=np.float64)
        src = np.ascontiguousarray(np.asarray(source, dtype=abi.SOURCE_DTYPE).reshape(1))
        arc = np.ascontiguousarray(np.asarray(() if arcs is None else arcs, dtype=np.float64).reshape(-1, 3))
        bands, states = np.zeros(24), np.zeros(6)
        n = lib().qmo_line_piece(self.handle, abi.ptr(rxy, C.c_int64), float(receiver_altitude_m), int(own_footprint),
                                 abi.ptr(pa, C.c_double), abi.ptr(pb, C.c_double), src.ctypes.data,
                                 int(arcs is None), abi.ptr(arc, C.c_double) if len(arc) else None, len(arc),
                                 abi.ptr(bands, C.c_double), abi.ptr(states, C.c_double))
        return bands.reshape(3, 8), states.reshape(2, 3), n

    def skyline_arcs(self, receiver_xy, lo_rad, hi_rad, radius_m, floor_m, cap=4096):
        """The (lo, hi, nearest) arcs the scene's skyline hands a lattice receiver for the wedge
        [lo_rad, hi_rad] (popup/src/obstacles/skyline.rs:39-110), in the order it visits them."""
        rxy = np.ascontiguousarray(receiver_xy, dtype=np.int64)
        out = np.zeros((cap, 3))
        n = lib().qmo_skyline_arcs(self.handle, abi.ptr(rxy, C.c_int64), float(lo_rad), float(hi_rad),
                                   float(radius_m), float(floor_m), abi.ptr(out, C.c_double), cap)
        assert n <= cap, n
        return out[:n].copy()

    def line_nodes(self, receiver_xy, start, end, floor_m):
        """A piece's quadrature nodes (start, end: metres relative to the receiver) with the wide
        buckets querying this scene's skyline from the lattice receiver above floor_m:
        (along_m, weight_rad, obstacles_on_ray) arrays, None for a degenerate piece."""
        rxy = np.ascontiguousarray(receiver_xy, dtype=np.int64)
        cap = 64 * 9 * 5
        along, weight = np.zeros(cap), np.zeros(cap)
        on_ray = np.zeros(cap, np.uint8)
        n = lib().qmo_scene_line_nodes(self.handle, abi.ptr(rxy, C.c_int64), float(floor_m),
                                       abi.ptr(_xyz(start), C.c_double), abi.ptr(_xyz(end), C.c_double),
                                       abi.ptr(along, C.c_double), abi.ptr(weight, C.c_double),
                                       abi.ptr(on_ray, C.c_uint8), cap)
        if n < 0:
            return None
        return along[:n], weight[:n], on_ray[:n].astype(bool)

    def enclosing(self, xy):
        xy = np.ascontiguousarray(np.asarray(xy).reshape(-1, 2), dtype=np.int64)
        out = np.zeros(len(xy), np.uint64)
        lib().qmo_enclosing_buildings(self.handle, abi.ptr(xy, C.c_int64), len(xy), abi.ptr(out, C.c_uint64),
                                      threads())
        return out

    def profile(self, frm, to, cap=65536):
        frm = np.ascontiguousarray(frm, dtype=np.int64)
        to = np.ascontiguousarray(to, dtype=np.int64)
        t, z, g = np.zeros(cap), np.zeros(cap), np.zeros(cap)
        h = np.zeros(1)
        n = lib().qmo_profile(self.handle, abi.ptr(frm, C.c_int64), abi.ptr(to, C.c_int64), abi.ptr(t, C.c_double),
                              abi.ptr(z, C.c_double), abi.ptr(g, C.c_double), cap, abi.ptr(h, C.c_double))
        return h[0], t[:n].copy(), z[:n].copy(), g[:n].copy()

    def evaluate_pairs(self, receiver_xy, receiver_altitude, own_footprint, point_of_receiver, source_of_pair,
                       receiver_of_pair, band_weight, n_points, nthreads=None):
        rxy = np.ascontiguousarray(np.asarray(receiver_xy).reshape(-1, 2), dtype=np.int64)
        ralt = _d(receiver_altitude)
        own = np.ascontiguousarray(own_footprint, dtype=np.uint64)
        por = np.ascontiguousarray(point_of_receiver, dtype=np.uint32)
        sop = np.ascontiguousarray(source_of_pair, dtype=np.uint32)
        rop = np.ascontiguousarray(receiver_of_pair, dtype=np.uint32)
        bw = None if band_weight is None else _d(band_weight)
        n = len(sop)
        sums = np.zeros((n, 9))
        bands = np.zeros((n, 3, 8))
        points = np.zeros((n_points, 6, 3, 8))
        lib().qmo_evaluate_pairs(self.handle, abi.ptr(rxy, C.c_int64), abi.ptr(ralt, C.c_double),
                                 abi.ptr(own, C.c_uint64), abi.ptr(por, C.c_uint32), len(rxy),
                                 abi.ptr(sop, C.c_uint32), abi.ptr(rop, C.c_uint32),
                                 abi.ptr(bw, C.c_double) if bw is not None else None, n,
                                 abi.ptr(sums, C.c_double), abi.ptr(bands, C.c_double), abi.ptr(points, C.c_double),
                                 n_points, nthreads or threads())
        return sums, bands, points

    def path_counts(self, frm, to):
        """Work counts of each pair's path [n][7]: crossings, profile vertices, diffraction
        candidates, and per state (homogeneous, favourable) the blocking candidates and hull
        points (receiver 4 m above its ground, source 0.05 m above its own)."""
        frm = np.ascontiguousarray(np.asarray(frm).reshape(-1, 2), dtype=np.int64)
        to = np.ascontiguousarray(np.asarray(to).reshape(-1, 2), dtype=np.int64)
        out = np.zeros((len(frm), 7))
        f = lib().qmo_path_counts
        for k in range(len(frm)):
            f(self.handle, abi.ptr(frm[k], C.c_int64), abi.ptr(to[k], C.c_int64), abi.ptr(out[k], C.c_double))
        return out

    def paint_grid(self, grid, cell_begin=0, cell_end=0, nthreads=None):
        """Per cell (of [cell_begin, cell_end), all when empty) the day band energies [n][8],
        the Lden-weighted A energy [n] and the number of edge tests."""
        g = abi.grid_desc(grid)
        n = (cell_end - cell_begin) if cell_end > cell_begin else grid.cells
        energy = np.zeros((n, 8))
        lden = np.zeros(n)
        tested = C.c_uint64()
        lib().qmo_paint_grid(self.handle, C.byref(g), cell_begin, cell_end, abi.ptr(energy, C.c_double),
                             abi.ptr(lden, C.c_double), nthreads or threads(), C.byref(tested))
        return energy, lden, tested.value

    def surrogate_samples(self, grid, cell_begin=0, cell_end=0, nthreads=None):
        """Surrogate features [rows][32], exact A_boundary labels [rows][8] (dB) and eligibility of
        every path of cells [cell_begin, cell_end) (all when empty) against the grid's sources
        (terrain scenes: two rows a path, homogeneous then favourable)."""
        g = abi.grid_desc(grid)
        if cell_end <= cell_begin:
            cell_begin, cell_end = 0, grid.cells
        n_src = (grid.source_end - grid.source_begin) if grid.source_end > grid.source_begin else len(self.scene.sources)
        rows = (cell_end - cell_begin) * n_src * (2 if self.scene.dem_altitude is not None else 1)
        f = np.zeros((rows, 32))
        lab = np.zeros((rows, 8))
        e = np.zeros(rows, np.uint8)
        lib().qmo_surrogate_samples(self.handle, C.byref(g), cell_begin, cell_end, abi.ptr(f, C.c_double),
                                    abi.ptr(lab, C.c_double), e.ctypes.data_as(C.POINTER(C.c_uint8)),
                                    nthreads or threads())
        return f, lab, e.astype(bool)


def zwicker(levels28):
    levels = _d(levels28)
    return lib().qmo_zwicker(abi.ptr(levels, C.c_double))


def zwicker_many(levels, nthreads=None):
    levels = _d(np.asarray(levels).reshape(-1, 28))
    out = np.zeros(len(levels))
    lib().qmo_zwicker_many(abi.ptr(levels, C.c_double), len(levels), abi.ptr(out, C.c_double),
                           nthreads or threads())
    return out


def level_histogram(levels, level_min, bin_db, n_bins):
    levels = _d(levels)
    counts = np.zeros(n_bins, np.uint32)
    lib().qmo_level_histogram(abi.ptr(levels, C.c_double), len(levels), level_min, bin_db, n_bins,
                              abi.ptr(counts, C.c_uint32))
    return counts


def level_bin(level, level_min, bin_db, n_bins):
    return lib().qmo_level_bin(level, level_min, bin_db, n_bins)


def percentile_table(n_rows=41):
    """The line-source quantile table by the reference's own seeded simulation
    (physics/src/percentile_tests.rs:1-102): float32 [n_rows][100]."""
    out = np.zeros((n_rows, 100), np.float32)
    lib().qmo_percentile_table(n_rows, abi.ptr(out, C.c_float))
    return out


def relative_intensity(lam, p):
    """The intensity, relative to its mean, a line of `lam` emitters per distance stays below with
    probability p (physics/src/percentile.rs:124-160); p a scalar or an array."""
    arr = np.ascontiguousarray(np.atleast_1d(np.asarray(p, dtype=np.float64)))
    out = np.zeros_like(arr)
    lib().qmo_relative_intensities(float(lam), abi.ptr(arr, C.c_double), len(arr), abi.ptr(out, C.c_double))
    return out if np.ndim(p) else float(out[0])


def ground_attenuation_bands(plane, source, receiver, g_path, g_impedance, g_floor, state):
    """A_ground per band over a mean plane (slope, intercept) (physics/src/cnossos/ground.rs)."""
    out = np.zeros(8)
    lib().qmo_ground_attenuation_bands(plane[0], plane[1], source[0], source[1], receiver[0], receiver[1], g_path,
                                       g_impedance, g_floor, state, abi.ptr(out, C.c_double))
    return out


def _pts(points):
    a = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 2))
    return a, abi.ptr(a, C.c_double) if len(a) else None


class StateRay:
    """A meteorological state's ray between source and receiver (physics/src/cnossos/
    rubber_band.rs:207-317): state 0 homogeneous, 1 favourable; radius_m None takes `between`'s."""

    def __init__(self, state, source, receiver, radius_m=None):
        self.state, self.radius = state, (radius_m or 0.0)
        self.source, _ = _pts(source)
        self.receiver, _ = _pts(receiver)

    def _ends(self):
        return abi.ptr(self.source, C.c_double), abi.ptr(self.receiver, C.c_double)

    def path_difference(self, start, points, end):
        p, pp = _pts(points)
        a, _ = _pts(start)
        b, _ = _pts(end)
        return lib().qmo_path_difference(self.state, self.radius, *self._ends(), abi.ptr(a, C.c_double), pp, len(p),
                                         abi.ptr(b, C.c_double))

    def diffraction_path(self, candidates):
        """(blocked, band points [(x, z)], blocking candidates [(x, z)]) (rubber_band.rs:373-444)."""
        c, cp = _pts(candidates)
        cap = max(len(c), 1)
        points, blocking = np.zeros((cap, 2)), np.zeros((cap, 2))
        n_points, n_blocking = C.c_size_t(), C.c_size_t()
        blocked = lib().qmo_diffraction_path(self.state, self.radius, *self._ends(), cp, len(c),
                                             abi.ptr(points, C.c_double), C.byref(n_points),
                                             abi.ptr(blocking, C.c_double), C.byref(n_blocking), cap)
        return (bool(blocked), [tuple(p) for p in points[:n_points.value]],
                [tuple(p) for p in blocking[:n_blocking.value]])

    def altitude(self, a, b, x):
        """The ray from a to b at x: chord altitude plus the arc's sag."""
        pa, _ = _pts(a)
        pb, _ = _pts(b)
        return lib().qmo_state_ray_altitude(self.state, self.radius, *self._ends(), abi.ptr(pa, C.c_double),
                                            abi.ptr(pb, C.c_double), float(x))


def _xyz(p):
    return np.ascontiguousarray(np.asarray(p, dtype=np.float64).reshape(3))


def line_geometry(start, end):
    """A straight piece seen from the receiver at the origin (physics/src/line.rs:86-124): dict of
    length, perpendicular, subtended angle and divergence factor; None under a millimetre."""
    out = np.zeros(4)
    if lib().qmo_line_geometry(abi.ptr(_xyz(start), C.c_double), abi.ptr(_xyz(end), C.c_double),
                               abi.ptr(out, C.c_double)) != 0:
        return None
    return dict(length_m=out[0], perpendicular_m=out[1], subtended_rad=out[2], divergence_factor=out[3])


def line_in_plane_angle_at(start, end, along_m):
    return lib().qmo_line_in_plane_angle_at(abi.ptr(_xyz(start), C.c_double), abi.ptr(_xyz(end), C.c_double),
                                            float(along_m))


def line_nodes(start, end, arcs=()):
    """A piece's quadrature nodes (physics/src/line.rs:180-355) given the arcs a skyline query
    hands over [(azimuth lo, azimuth hi, nearest range)]: (along_m, weight_rad, obstacles_on_ray)
    arrays."""
    a = np.ascontiguousarray(np.asarray(arcs, dtype=np.float64).reshape(-1, 3))
    cap = 64 * 9 * 5
    along, weight = np.zeros(cap), np.zeros(cap)
    on_ray = np.zeros(cap, np.uint8)
    n = lib().qmo_line_nodes(abi.ptr(_xyz(start), C.c_double), abi.ptr(_xyz(end), C.c_double),
                             abi.ptr(a, C.c_double) if len(a) else None, len(a), abi.ptr(along, C.c_double),
                             abi.ptr(weight, C.c_double), abi.ptr(on_ray, C.c_uint8), cap)
    if n < 0:
        return None
    return along[:n], weight[:n], on_ray[:n].astype(bool)


def favourable_at(row, azimuth_rad):
    """p of a period's 16-sector row (float, as a scene stores it) along an azimuth
    (physics/src/weather.rs:61-70)."""
    r = np.ascontiguousarray(np.asarray(row, dtype=np.float32).reshape(16))
    return lib().qmo_favourable_at(abi.ptr(r, C.c_float), float(azimuth_rad))


def nden_cell(sone):
    """The map cell of a loudness (paint/src/levels.rs:25-33)."""
    return int(lib().qmo_nden_cell(float(sone)))


def lden_cell(energy):
    """The map cell of a linear Lden energy (paint/src/levels.rs:87-98); ValueError where the
    reference returns its error."""
    c = lib().qmo_lden_cell(float(energy))
    if c < 0:
        raise ValueError(f"invalid Lden energy {energy}")
    return c


HM3_TILE_PX = 512
HM3_STREAM_BYTES = 6 + HM3_TILE_PX * HM3_TILE_PX


def hm3_predict(cells, layer, metric):
    """One tile's HM3 / HMD stream before Brotli (paint/src/hm3.rs:95-109): uint8 [6 + 512^2]."""
    c = np.ascontiguousarray(np.asarray(cells, dtype=np.uint8).reshape(HM3_TILE_PX * HM3_TILE_PX))
    out = np.zeros(HM3_STREAM_BYTES, np.uint8)
    if lib().qmo_hm3_predict(abi.ptr(c, C.c_uint8), int(layer), int(metric), abi.ptr(out, C.c_uint8)) != 0:
        raise ValueError(f"unknown HM3 layer {layer}")
    return out


def hm3_unpredict(residuals):
    """The Paeth residuals of a stream (its bytes after the 6-byte head) back to the cells
    (paint/src/hm3.rs:162-165): uint8 [512][512]."""
    r = np.array(np.asarray(residuals, dtype=np.uint8).reshape(HM3_TILE_PX * HM3_TILE_PX), copy=True)
    lib().qmo_hm3_unpredict(abi.ptr(r, C.c_uint8))
    return r.reshape(HM3_TILE_PX, HM3_TILE_PX)


def quantize_cells(lden_energy, sone=None, assessed=None):
    """Map cells of pixels (paint/src/levels.rs:55-111): (lden_cells [n][7], nden_cells [n][7] or
    None); ValueError naming the first invalid pixel and layer, as the reference's error does."""
    e = np.ascontiguousarray(np.asarray(lden_energy, dtype=np.float64).reshape(-1, abi.LAYERS))
    n = len(e)
    s = None if sone is None else np.ascontiguousarray(np.asarray(sone, dtype=np.float64).reshape(n, abi.LAYERS + 1))
    a = None if assessed is None else np.ascontiguousarray(np.asarray(assessed, dtype=np.uint8).reshape(n))
    lc = np.zeros((n, abi.LAYERS + 1), np.uint8)
    nc = None if s is None else np.zeros((n, abi.LAYERS + 1), np.uint8)
    bad = lib().qmo_quantize_cells(abi.ptr(e, C.c_double), abi.ptr(s, C.c_double), abi.ptr(a, C.c_uint8), n,
                                   abi.ptr(lc, C.c_uint8), abi.ptr(nc, C.c_uint8))
    if bad >= 0:
        pixel, layer = divmod(int(bad), 8)
        where = f"layer {layer}" if layer < abi.LAYERS else "total"
        raise ValueError(f"pixel {pixel}, {where}: invalid Lden energy")
    return lc, nc


# ---------------------------------------------------------------------------------------------
# Doc 29 (physics/src/doc29/{npd,corrections,segment}.rs)

def lateral_attenuation_db(height_m, lateral_m):
    return lib().qmo_lateral_attenuation_db(height_m, lateral_m)


def speed_correction_db(v_ref_kt, speed_kt):
    return lib().qmo_speed_correction_db(v_ref_kt, speed_kt)


def finite_segment_energy_fraction(along_m, length_m, scaled_m):
    return lib().qmo_finite_segment_energy_fraction(along_m, length_m, scaled_m)


def installation_energy_gain(installation, height_m, slant_m):
    return lib().qmo_installation_energy_gain(installation, height_m, slant_m)


def npd_level(curve10, slant_m, tail_alpha):
    c = _d(curve10)
    return lib().qmo_npd_level(abi.ptr(c, C.c_double), slant_m, tail_alpha)


def tail_absorption(sel10):
    c = _d(sel10)
    return lib().qmo_tail_absorption(abi.ptr(c, C.c_double))


def flight_grid(flights, cell_begin=0, cell_end=0, grid=None, nthreads=None):
    """Per cell of [cell_begin, cell_end): (LAE [n], thirds [n][28], sone [n])."""
    g = abi.flight_grid_desc(grid or flights.grid)
    n = (cell_end - cell_begin) if cell_end > cell_begin else g.nx * g.ny
    types = np.ascontiguousarray(flights.types, dtype=abi.AIRCRAFT_TYPE_DTYPE)
    segs = np.ascontiguousarray(flights.segments, dtype=abi.FLIGHT_SEGMENT_DTYPE)
    lae, thirds, sone = np.zeros(n), np.zeros((n, 28)), np.zeros(n)
    lib().qmo_flight_grid(types.ctypes.data, len(types), segs.ctypes.data, len(segs), C.byref(g), cell_begin,
                          cell_end, abi.ptr(lae, C.c_double), abi.ptr(thirds, C.c_double), abi.ptr(sone, C.c_double),
                          nthreads or threads())
    return lae, thirds, sone


# ---------------------------------------------------------------------------------------------
# Aircraft boxes (physics/src/doc29/{box_sums,boxes,screening}.rs, popup/src/aircraft/{boxes,horizons}.rs,
# paint/src/flight_boxes.rs)

def path_difference_loss_db(delta_m):
    return lib().qmo_path_difference_loss_db(delta_m)


def edge_loss_db(edge_range_m, edge_height_m, source_range_m, source_height_m):
    return lib().qmo_edge_loss_db(edge_range_m, edge_height_m, source_range_m, source_height_m)


def screened_sel_db(free_db, lateral_db, terrain_db, building_db):
    return lib().qmo_screened_sel_db(free_db, lateral_db, terrain_db, building_db)


def flight_weight(kind, distance_m, coarse_m):
    return lib().qmo_flight_weight(kind, distance_m, coarse_m)


def horizon_loss_db(floats, sectors, point_m):
    f = np.ascontiguousarray(floats, dtype=np.float32)
    p = _d(point_m)
    return lib().qmo_horizon_loss_db(abi.ptr(f, C.c_float), sectors, abi.ptr(p, C.c_double))


def segment_sel_db(aircraft_type, segment, receiver_m):
    t = np.ascontiguousarray(np.atleast_1d(aircraft_type), dtype=abi.AIRCRAFT_TYPE_DTYPE)
    g = np.ascontiguousarray(np.atleast_1d(segment), dtype=abi.FLIGHT_SEGMENT_DTYPE)
    rx, ry, rz = (float(v) for v in receiver_m)
    return lib().qmo_segment_sel_db(t.ctypes.data, g.ctypes.data, rx, ry, rz)


def box_sums(types, pieces, period_weights):
    """The box of `pieces` (FLIGHT_SEGMENT_DTYPE, each of types[piece.type]) weighted per period by
    period_weights [n][3], as the builder closes it; None for a box without energy."""
    t = np.ascontiguousarray(types, dtype=abi.AIRCRAFT_TYPE_DTYPE)
    g = np.ascontiguousarray(np.atleast_1d(pieces), dtype=abi.FLIGHT_SEGMENT_DTYPE)
    w = _d(np.asarray(period_weights, dtype=np.float64).reshape(len(g), 3))
    out = np.zeros(1, dtype=abi.FLIGHT_BOX_DTYPE)
    if not lib().qmo_box_sums(t.ctypes.data, g.ctypes.data, len(g), abi.ptr(w, C.c_double), out.ctypes.data):
        return None
    return out[0]


def box_sel(box, point, horizons=None):
    """(sel_energy [3], installation fractions [3][3]) of one box at one point."""
    b = np.ascontiguousarray(np.atleast_1d(box), dtype=abi.FLIGHT_BOX_DTYPE)
    p = np.ascontiguousarray(np.atleast_1d(point), dtype=abi.FLIGHT_POINT_DTYPE)
    h = None if horizons is None else np.ascontiguousarray(horizons, dtype=np.float32)
    sel, fractions = np.zeros(3), np.zeros((3, 3))
    lib().qmo_box_sel(b.ctypes.data, p.ctypes.data, None if h is None else abi.ptr(h, C.c_float),
                      abi.ptr(sel, C.c_double), abi.ptr(fractions, C.c_double))
    return sel, fractions


def flight_sums(boxes, points, horizons, segments, n_sums, nthreads=None):
    """sums [n_sums][FLIGHT_SUMS] of every request band and the number of boxes heard."""
    b = np.ascontiguousarray(boxes, dtype=abi.FLIGHT_BOX_DTYPE)
    p = np.ascontiguousarray(points, dtype=abi.FLIGHT_POINT_DTYPE)
    h = None if horizons is None else np.ascontiguousarray(horizons, dtype=np.float32)
    s = np.ascontiguousarray(segments, dtype=abi.BOX_SEGMENT_DTYPE)
    sums = np.zeros((n_sums, abi.FLIGHT_SUMS))
    heard = lib().qmo_flight_sums(b.ctypes.data, p.ctypes.data, None if h is None else abi.ptr(h, C.c_float),
                                  s.ctypes.data, len(s), abi.ptr(sums, C.c_double), n_sums, nthreads or threads())
    return sums, heard
