// Rays from points off the integer lattice: a line piece's quadrature nodes lie anywhere along the
// piece (physics/src/line.rs:178-206), so each node's ray starts at a fractional position. The
// reference's walks take f64 step coordinates (popup/src/obstacles/crossings.rs:13-28, 163-226;
// popup/src/scene.rs:242-296); these are the same walks in double, each product and sum rounded
// on its own (no contraction), so a node's crossings and ground profile are the reference's. On
// lattice ends they agree with the integer walks of qm_path.cuh.
#pragma once

#include "qm_path.cuh"

namespace qm {

// The ground and ground factor at a position (steps): bilinear between the four DEM nodes around it,
// clamped to the DEM (popup/src/scene.rs:182-200).
__device__ inline void terrain_at_d(const SceneDev &S, double x, double y, double &z, double &g) {
    if (S.dem_nx == 0) {
        z = S.flat_z;
        g = S.flat_g;
        return;
    }
    double fx = __ddiv_rn(__dsub_rn(x, (double)S.dem_ox), (double)S.dem_sp);
    double fy = __ddiv_rn(__dsub_rn(y, (double)S.dem_oy), (double)S.dem_sp);
    fx = fmin(fmax(fx, 0.0), (double)(S.dem_nx - 1));
    fy = fmin(fmax(fy, 0.0), (double)(S.dem_ny - 1));
    const long long i0 = min((long long)floor(fx), (long long)S.dem_nx - 2);
    const long long j0 = min((long long)floor(fy), (long long)S.dem_ny - 2);
    const double ax = __dsub_rn(fx, (double)i0), ay = __dsub_rn(fy, (double)j0);
    const float2 *row0 = S.dem + j0 * S.dem_nx, *row1 = row0 + S.dem_nx;
    const float2 p = __ldg(row0 + i0), q = __ldg(row0 + i0 + 1), r = __ldg(row1 + i0), u = __ldg(row1 + i0 + 1);
    auto bil = [&](double a, double b, double c, double d) {
        const double lo = __dadd_rn(a, __dmul_rn(ax, __dsub_rn(b, a)));
        const double hi = __dadd_rn(c, __dmul_rn(ax, __dsub_rn(d, c)));
        return __dadd_rn(lo, __dmul_rn(ay, __dsub_rn(hi, lo)));
    };
    z = bil(p.x, q.x, r.x, u.x);
    g = bil(p.y, q.y, r.y, u.y);
}

// The ground profile under a ray from a fractional start to a lattice receiver (the oracle's and
// the reference's f64 walk): the start, a vertex wherever the ray crosses a DEM row or column line
// strictly inside (a row first at a tie), the end. The same interface as TerrainWalk.
struct TerrainWalkD {
    double sx, sy, dx, dy, sp, next_col, next_row, col_step, row_step;
    float length;
    bool dem;
    int stage;
    float2 start_zg, end_zg;

    __device__ void init(const SceneDev &S, double x0, double y0, double x1, double y1, float length_m) {
        sx = x0;
        sy = y0;
        dx = __dsub_rn(x1, x0);
        dy = __dsub_rn(y1, y0);
        length = length_m;
        dem = S.dem_nx != 0;
        stage = 0;
        double z, g;
        terrain_at_d(S, x0, y0, z, g);
        start_zg = make_float2((float)z, (float)g);
        terrain_at_d(S, x1, y1, z, g);
        end_zg = make_float2((float)z, (float)g);
        if (!dem) return;
        sp = (double)S.dem_sp;
        const double cx = __ddiv_rn(__dsub_rn(sx, (double)S.dem_ox), sp), cy = __ddiv_rn(__dsub_rn(sy, (double)S.dem_oy), sp);
        next_col = dx > 0 ? floor(cx) + 1.0 : ceil(cx) - 1.0;
        next_row = dy > 0 ? floor(cy) + 1.0 : ceil(cy) - 1.0;
        col_step = dx > 0 ? 1.0 : -1.0;
        row_step = dy > 0 ? 1.0 : -1.0;
    }

    __device__ __forceinline__ bool next(const SceneDev &S, TV &v) {
        if (stage == 0) {
            stage = dem ? 1 : 2;
            v = TV{0.0f, start_zg.x, start_zg.y};
            return true;
        }
        if (stage == 1) {
            const double t_col = dx != 0.0 ? __ddiv_rn(__dsub_rn(__dadd_rn((double)S.dem_ox, __dmul_rn(next_col, sp)), sx), dx) : INFINITY;
            const double t_row = dy != 0.0 ? __ddiv_rn(__dsub_rn(__dadd_rn((double)S.dem_oy, __dmul_rn(next_row, sp)), sy), dy) : INFINITY;
            const double t = fmin(t_col, t_row);
            if (t < 1.0) {
                if (t_row <= t_col) {
                    const double px = __dadd_rn(sx, __dmul_rn(t, dx));
                    const double fx = __ddiv_rn(__dsub_rn(px, (double)S.dem_ox), sp);
                    const double i0 = floor(fx), f = __dsub_rn(fx, i0);
                    const float2 a = dem_node(S, (int)i0, (int)next_row), b = dem_node(S, (int)i0 + 1, (int)next_row);
                    v = TV{(float)t * length, (float)__dadd_rn((double)a.x, __dmul_rn(f, __dsub_rn((double)b.x, (double)a.x))),
                           (float)__dadd_rn((double)a.y, __dmul_rn(f, __dsub_rn((double)b.y, (double)a.y)))};
                    next_row += row_step;
                } else {
                    const double py = __dadd_rn(sy, __dmul_rn(t, dy));
                    const double fy = __ddiv_rn(__dsub_rn(py, (double)S.dem_oy), sp);
                    const double j0 = floor(fy), f = fmin(fmax(__dsub_rn(fy, j0), 0.0), 1.0);
                    const float2 a = dem_node(S, (int)next_col, (int)j0), b = dem_node(S, (int)next_col, (int)j0 + 1);
                    v = TV{(float)t * length, (float)__dadd_rn((double)a.x, __dmul_rn(f, __dsub_rn((double)b.x, (double)a.x))),
                           (float)__dadd_rn((double)a.y, __dmul_rn(f, __dsub_rn((double)b.y, (double)a.y)))};
                    next_col += col_step;
                }
                return true;
            }
            stage = 2;
        }
        if (stage == 2) {
            stage = 3;
            v = TV{length, end_zg.x, end_zg.y};
            return true;
        }
        return false;
    }
};

__device__ __forceinline__ void start_walk(TerrainWalkD &walk, const SceneDev &S, double sxd, double syd, int, int,
                                           int rx, int ry, float L) {
    walk.init(S, sxd, syd, (double)rx, (double)ry, L);
}

// Whether an edge hit enters or leaves its ring (crossings.rs:80-111), in double from a fractional
// start.
__device__ __noinline__ bool edge_bounds_roof_d(const SceneDev &S, double sx, double sy, double dx, double dy,
                                                uint32_t edge, uint32_t first, uint32_t count) {
    auto side = [&](uint32_t index) {
        const int2 v = S.vertices[index];
        return __dsub_rn(__dmul_rn(dx, __dsub_rn((double)v.y, sy)), __dmul_rn(dy, __dsub_rn((double)v.x, sx)));
    };
    const double a = side(edge), b = side(edge + 1);
    if (a != 0.0 && b != 0.0) return true;
    const uint32_t distinct = count - 1;
    const uint32_t vertex = ((a == 0.0 ? edge : edge + 1) - first) % distinct;
    double n0 = 0.0, n1 = 0.0;
    for (uint32_t offset = 1; offset < distinct; ++offset) {
        if (n0 == 0.0) n0 = side(first + (vertex + distinct - offset) % distinct);
        if (n1 == 0.0) n1 = side(first + (vertex + offset) % distinct);
        if (n0 != 0.0 && n1 != 0.0) break;
    }
    return n0 * n1 < 0.0;
}

// Every crossing of the segment from the fractional point (sx, sy) to the point (rx, ry) (a lattice
// point for a path, fractional for a horizon's ray)
// with an obstacle edge (crossings.rs:163-226 in f64): the cells the segment passes in order, and
// in each cell the edges whose box meets the segment's piece in the cell (padded by 1e-9 of the
// segment's size), each tested by segment_intersection_t (crossings.rs:13-28); then sorted and
// deduplicated as list_crossings does, without the receiver's own walls.
template <int MAXC>
__device__ int list_crossings_d(const SceneDev &S, double sx, double sy, double rx, double ry, uint32_t rcv_own,
                                XRec *xs, uint32_t &status, uint32_t &edges_tested) {
    int n = 0;
    const double ex_ = rx, ey_ = ry;
    const double d0 = __dsub_rn(ex_, sx), d1 = __dsub_rn(ey_, sy);
    const double cs = (double)S.cell_steps;
    long long cell[2] = {(long long)floor(__ddiv_rn(sx, cs)), (long long)floor(__ddiv_rn(sy, cs))};
    const long long last[2] = {(long long)floor(__ddiv_rn(ex_, cs)), (long long)floor(__ddiv_rn(ey_, cs))};
    const long long step[2] = {d0 >= 0.0 ? 1 : -1, d1 >= 0.0 ? 1 : -1};
    const double start[2] = {sx, sy}, delta[2] = {d0, d1};
    double t_delta[2], t_max[2];
    for (int axis = 0; axis < 2; ++axis) {
        t_delta[axis] = delta[axis] != 0.0 ? fabs(__ddiv_rn(cs, delta[axis])) : INFINITY;
        if (delta[axis] == 0.0) {
            t_max[axis] = INFINITY;
        } else {
            const double boundary = __dmul_rn((double)(cell[axis] + (delta[axis] >= 0.0 ? 1 : 0)), cs);
            t_max[axis] = fabs(__ddiv_rn(__dsub_rn(boundary, start[axis]), delta[axis]));
        }
    }
    const double pad = __dmul_rn(1e-9, __dadd_rn(__dadd_rn(1.0, fabs(d0)), fabs(d1)));
    double t_enter = 0.0;
    const int guard_max = (int)(llabs(last[0] - cell[0]) + llabs(last[1] - cell[1])) + 2;
    for (int guard = 0; guard < guard_max; ++guard) {
        if (cell[0] >= 0 && cell[1] >= 0 && cell[0] < S.cells_x && cell[1] < S.cells_y) {
            const uint2 range = __ldg(S.cell_range + cell[1] * S.cells_x + cell[0]);
            if (range.x < range.y) {
                const double t_exit = fmin(fmin(t_max[0], t_max[1]), 1.0);
                const double ta = fmin(fmax(t_enter, 0.0), 1.0), tb = fmin(fmax(t_exit, 0.0), 1.0);
                const double px = __dadd_rn(sx, __dmul_rn(d0, ta)), py = __dadd_rn(sy, __dmul_rn(d1, ta));
                const double qx = __dadd_rn(sx, __dmul_rn(d0, tb)), qy = __dadd_rn(sy, __dmul_rn(d1, tb));
                const long long low0 = (long long)floor(__dsub_rn(fmin(px, qx), pad));
                const long long low1 = (long long)floor(__dsub_rn(fmin(py, qy), pad));
                const long long high0 = (long long)ceil(__dadd_rn(fmax(px, qx), pad));
                const long long high1 = (long long)ceil(__dadd_rn(fmax(py, qy), pad));
                for (uint32_t k = range.x; k < range.y; ++k) {
                    const int4 seg = __ldg(S.cell_seg + k);
                    if (!(high0 >= min(seg.x, seg.z) && max(seg.x, seg.z) >= low0 && high1 >= min(seg.y, seg.w) &&
                          max(seg.y, seg.w) >= low1))
                        continue;
                    ++edges_tested;
                    const double ex = (double)(seg.z - seg.x), ey = (double)(seg.w - seg.y);
                    const double den = __dsub_rn(__dmul_rn(d0, ey), __dmul_rn(d1, ex));
                    if (den == 0.0) continue;
                    const double wx = __dsub_rn((double)seg.x, sx), wy = __dsub_rn((double)seg.y, sy);
                    const double t = __ddiv_rn(__dsub_rn(__dmul_rn(wx, ey), __dmul_rn(wy, ex)), den);
                    const double u = __ddiv_rn(__dsub_rn(__dmul_rn(wx, d1), __dmul_rn(wy, d0)), den);
                    if (!(t > 0.0 && t < 1.0 && u >= 0.0 && u <= 1.0)) continue;
                    const uint2 ref = __ldg(S.cell_ref + k);
                    bool repeat = false;
                    for (int j = n - 1; j >= 0 && j >= n - 4; --j) repeat |= xs[j].edge == ref.x;
                    if (repeat) continue;
                    if (n >= MAXC) {
                        status |= FAILED_CAPACITY;
                        return n;
                    }
                    const OutlineDev o = S.outlines[ref.y];
                    const bool building = o.building != 0;
                    const bool bounds = building && edge_bounds_roof_d(S, sx, sy, d0, d1, ref.x, o.first, o.count);
                    xs[n++] = XRec{t, ref.x, ref.y | (building ? X_BUILDING : 0u) | (bounds ? X_BOUNDS : 0u), o.height, o.fp};
                }
            }
        }
        if (cell[0] == last[0] && cell[1] == last[1]) break;
        t_enter = fmin(t_max[0], t_max[1]);
        int axis;
        if (cell[0] == last[0])
            axis = 1;
        else if (cell[1] == last[1] || t_max[0] < t_max[1])
            axis = 0;
        else
            axis = 1;
        t_max[axis] = __dadd_rn(t_max[axis], t_delta[axis]);
        cell[axis] += step[axis];
    }
    return finish_crossings(S, xs, n, rcv_own);
}

}  // namespace qm
