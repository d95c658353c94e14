// The receiver skyline of the line quadrature (popup/src/obstacles/skyline.rs:22-110): the
// obstacle edges near a receiver, each as its azimuth arc and nearest horizontal range.
//
// The index follows the reference's tile cells in the reference's own frame: lattice steps with
// y growing south, so a scene point (x, y) (y north) is (x, -y) there; cells of 256 steps; each
// edge listed in every cell its supercover walk passes through (tiles/src/obstacles/cells.rs:
// 13-47), consecutive edges of one outline in one run, and per cell the height of its tallest
// outline (popup/src/obstacles/tile.rs:93-104). It is flat arrays, the same on the host and in
// device memory: the occupied cells' keys sorted row-major, their run ranges and tallest
// heights, and the runs. The query is __host__ __device__ and allocates nothing.
#pragma once

#include <cuda_runtime.h>

#include <math.h>
#include <stdint.h>

#include "../../include/qm_batch.h"
#include "qm_line.cuh"

namespace qm {
namespace skyline {

constexpr int64_t CELL_STEPS = 256;

struct Run {
    uint32_t outline, first_edge, count;
};

// Views of an index's arrays and of the scene outlines it lists.
struct Index {
    const uint64_t *keys;       // [n_cells], ascending (row-major, see cell_key)
    const uint32_t *run_start;  // [n_cells + 1]: a cell's runs are runs[run_start[c] .. run_start[c+1])
    const float *tallest;       // [n_cells]: the tallest outline listed in the cell, metres
    const Run *runs;
    const int32_t *vertices;    // the scene's [n][2] steps, y north
    const qm_outline *outlines;
    uint32_t n_cells;
    double step_m;
};

// Row-major keys that sort as (row, column) for negative cells too: each signed 32-bit index
// with its sign bit flipped, the row above the column.
__host__ __device__ inline uint64_t cell_key(int64_t column, int64_t row) {
    return ((uint64_t)((uint32_t)(int32_t)row ^ 0x80000000u) << 32) | (uint64_t)((uint32_t)(int32_t)column ^ 0x80000000u);
}

__host__ __device__ inline int64_t floor_div(int64_t a, int64_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// The cells the edge (sx, sy) -> (ex, ey) (reference frame) passes through, 4-connected in
// walking order; a tie steps the row, and the walk never leaves the box of its end cells
// (cells.rs:13-47). visit(column, row) per cell.
#pragma nv_exec_check_disable
template <class Visit>
__host__ __device__ void edge_cells(int64_t sx, int64_t sy, int64_t ex, int64_t ey, Visit &visit) {
    int64_t cell[2] = {floor_div(sx, CELL_STEPS), floor_div(sy, CELL_STEPS)};
    const int64_t last[2] = {floor_div(ex, CELL_STEPS), floor_div(ey, CELL_STEPS)};
    const double delta[2] = {(double)(ex - sx), (double)(ey - sy)};
    const int64_t start[2] = {sx, sy};
    int64_t step[2];
    double t_delta[2], t_max[2];
    for (int axis = 0; axis < 2; ++axis) {
        step[axis] = delta[axis] >= 0.0 ? 1 : -1;
        if (delta[axis] == 0.0) {
            t_delta[axis] = INFINITY;
            t_max[axis] = INFINITY;
        } else {
            t_delta[axis] = fabs((double)CELL_STEPS / delta[axis]);
            const int64_t boundary = (cell[axis] + (delta[axis] >= 0.0 ? 1 : 0)) * CELL_STEPS;
            t_max[axis] = fabs((double)(boundary - start[axis]) / delta[axis]);
        }
    }
    for (;;) {
        visit(cell[0], cell[1]);
        if (cell[0] == last[0] && cell[1] == last[1]) return;
        int axis;
        if (cell[0] == last[0])
            axis = 1;
        else if (cell[1] == last[1] || t_max[0] < t_max[1])
            axis = 0;
        else
            axis = 1;
        t_max[axis] += t_delta[axis];
        cell[axis] += step[axis];
    }
}

// The first index whose key is not below `key`.
__host__ __device__ inline uint32_t lower_bound(const uint64_t *keys, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Every arc the receiver at scene steps (rx, ry) gets for the wedge [lo, hi] within radius_m:
// cells beyond the radius or wholly on the far side of either wedge edge are skipped, so are
// cells whose tallest outline, and walls whose own height, stay at or under floor_m (the sight
// line's height); an edge through the receiver gives nothing (skyline.rs:39-110).
// visit(arc_lo, arc_hi, nearest) in row, column, run order, once per cell an edge is listed in.
#pragma nv_exec_check_disable
template <class Visit>
__host__ __device__ void arcs(const Index &ix, int64_t rx, int64_t ry, double lo, double hi, double radius_m,
                              double floor_m, Visit &visit) {
    const double m = ix.step_m, cs = (double)CELL_STEPS;
    const double ox = (double)rx, oy = -(double)ry;
    const double low[2] = {cos(lo), sin(lo)}, high[2] = {cos(hi), sin(hi)};
    if (ix.n_cells == 0 || !(radius_m >= 0.0)) return;
    // The cells within the radius's box, held to the rows the index occupies and to 32-bit
    // indices (which changes nothing a query visits, and bounds the walk for any radius).
    auto cell_of = [&](double steps) { return (int64_t)fmin(fmax(floor(steps / cs), (double)INT32_MIN), (double)INT32_MAX); };
    const int64_t first_row = (int64_t)(int32_t)((uint32_t)(ix.keys[0] >> 32) ^ 0x80000000u);
    const int64_t last_row = (int64_t)(int32_t)((uint32_t)(ix.keys[ix.n_cells - 1] >> 32) ^ 0x80000000u);
    int64_t row0 = cell_of(oy - radius_m / m), row1 = cell_of(oy + radius_m / m);
    row0 = row0 > first_row ? row0 : first_row;
    row1 = row1 < last_row ? row1 : last_row;
    const int64_t col0 = cell_of(ox - radius_m / m), col1 = cell_of(ox + radius_m / m);
    for (int64_t row = row0; row <= row1; ++row) {
        const double south = (oy - (double)(row + 1) * cs) * m, north = (oy - (double)row * cs) * m;
        const double dy = fmax(fmax(south, -north), 0.0);
        const uint64_t end_key = cell_key(col1, row);
        for (uint32_t c = lower_bound(ix.keys, ix.n_cells, cell_key(col0, row)); c < ix.n_cells && ix.keys[c] <= end_key;
             ++c) {
            const int64_t column = (int64_t)(int32_t)((uint32_t)ix.keys[c] ^ 0x80000000u);
            const double west = ((double)column * cs - ox) * m, east = ((double)(column + 1) * cs - ox) * m;
            const double dx = fmax(fmax(west, -east), 0.0);
            if (dx * dx + dy * dy > radius_m * radius_m) continue;
            const double corners[4][2] = {{west, south}, {east, south}, {west, north}, {east, north}};
            bool below = true, above = true;
            for (int k = 0; k < 4; ++k) {
                below = below && low[0] * corners[k][1] - low[1] * corners[k][0] < 0.0;
                above = above && corners[k][0] * high[1] - corners[k][1] * high[0] < 0.0;
            }
            if (below || above) continue;
            if ((double)ix.tallest[c] <= floor_m) continue;
            for (uint32_t r = ix.run_start[c]; r < ix.run_start[c + 1]; ++r) {
                const Run run = ix.runs[r];
                const qm_outline &rec = ix.outlines[run.outline];
                if (rec.building == 0 && (double)rec.height_m <= floor_m) continue;
                const size_t first = (size_t)rec.first_vertex + run.first_edge;
                double a[2] = {((double)ix.vertices[2 * first] - ox) * m, (oy + (double)ix.vertices[2 * first + 1]) * m};
                double azimuth_a = atan2(a[1], a[0]);
                for (size_t v = first + 1; v <= first + run.count; ++v) {
                    const double b[2] = {((double)ix.vertices[2 * v] - ox) * m, (oy + (double)ix.vertices[2 * v + 1]) * m};
                    const double azimuth_b = atan2(b[1], b[0]);
                    // The edge's nearest point to the receiver (skyline.rs:9-20).
                    const double ex = b[0] - a[0], ey = b[1] - a[1], length2 = ex * ex + ey * ey;
                    const double t = length2 > 0.0 ? fmin(fmax(-(a[0] * ex + a[1] * ey) / length2, 0.0), 1.0) : 0.0;
                    const double px = a[0] + t * ex, py = a[1] + t * ey;
                    const double nearest = sqrt(px * px + py * py);
                    if (nearest >= 1e-6 && nearest <= radius_m) {
                        const double unwrapped_b = azimuth_a + line::wrap_to_pi(azimuth_b - azimuth_a);
                        visit(fmin(azimuth_a, unwrapped_b), fmax(azimuth_a, unwrapped_b), nearest);
                    }
                    a[0] = b[0];
                    a[1] = b[1];
                    azimuth_a = azimuth_b;
                }
            }
        }
    }
}

}  // namespace skyline
}  // namespace qm
