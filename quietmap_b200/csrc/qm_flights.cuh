// A square's aircraft boxes summed at lattice points (include/qm_flights.h), FP64 throughout.
//
// Boxes are decoded once into BoxDev records (what box_sel_at_receiver derives from a box alone).
// The sums kernel takes one request band (a `sum`) per CTA slice: its segments' box reads are
// flattened and strided over the CTA's threads, each thread reading its boxes by the click-time
// equation (physics/src/doc29/boxes.rs:156-280) through the point's horizons (staged in shared
// memory once per slice), the lattice weight (paint/src/flight_boxes.rs:24-33) and the reach
// (popup/src/aircraft/boxes.rs:272-316). Pass classes (popup/src/aircraft.rs:86-95) gather in
// shared memory, the period energies in registers; a slice adds its totals to the request band's
// sums once at its end.
#pragma once

#include <math_constants.h>

#include <cstdint>

#include "../../include/qm_flights.h"

namespace qm {
namespace fl {

constexpr int ND = QM_NPD_DISTANCES;
constexpr int CLASSES = QM_PASS_CLASSES;
constexpr int THREADS = 128;
// Box reads a CTA slice takes at most: enough to amortise its horizon staging and class flush.
constexpr uint64_t SLICE_READS = 2048;
constexpr double METRES_PER_FOOT = 0.3048;                    // npd.rs:17
constexpr double NPD_NEAREST_SLANT_M = 100.0 * METRES_PER_FOOT;  // npd.rs:26
constexpr double NPD_LAST_DISTANCE_M = 25000.0 * METRES_PER_FOOT;  // npd.rs:28
constexpr double TAIL_ANCHOR_M = 16000.0;                     // npd.rs:330
constexpr double SHARE_NEAR_M = 1000.0 * METRES_PER_FOOT;    // box_sums.rs:14
constexpr double SHARE_FAR_M = TAIL_ANCHOR_M;
constexpr double PATH_DIFFERENCE_SLOPE_PER_M = 29.2;          // screening.rs:8
constexpr double GRAZING_LOSS_DB = 4.771212547196624;         // screening.rs:10
constexpr double SCREENING_CAP_DB = 18.0;                     // screening.rs:12
constexpr double SCREENING_CEILING_M = 7620.0;                // screening.rs:15
constexpr double PI_D = 3.141592653589793116;
constexpr double TAU_D = 6.283185307179586232;
constexpr double LN10_D = 2.302585092994045684;

// A box as the sums kernel reads it: the position first (the reach test reads only those), then
// what the click-time equation reads. 624 bytes, 16-byte aligned.
struct __align__(16) BoxDev {
    double east, north, centroid_alt, ground;
    double sin_axis, cos_axis, gradient, spread;
    double average_length, pad0;
    double piece_length[3];
    double passing[3];
    double levels[3][ND];
    double tail[3];
    double lg_scaled[ND];
    double shares[3][2][3];
    uint32_t helicopter, silent;  // silent: bit p set when period p's levels are all -inf
};
static_assert(sizeof(BoxDev) == 624, "BoxDev layout");

// log10 of the NPD distances in feet, taken on the host by the cores' log10 (npd.rs:115-150).
struct NpdLogs {
    double lg[ND];
    double lg_share_span;   // log10 of the installation shares' far slant over their near one
    double tail_anchor_db;  // 20 log10 of the tail anchor over 25,000 ft
};

// One copy each of the FP64 functions the equation calls at many sites: inlined at every site,
// the equation's code overflowed the instruction cache and its warps waited on instruction fetch.
__device__ __noinline__ double f_exp(double x) { return exp(x); }
__device__ __noinline__ double f_log10(double x) { return log10(x); }
__device__ __noinline__ double f_atan(double x) { return atan(x); }
__device__ __noinline__ double f_hypot(double x, double y) { return hypot(x, y); }
__device__ __noinline__ double f_pow(double x, double y) { return pow(x, y); }

__device__ __forceinline__ double energy_of(double level_db) { return f_exp(level_db * (LN10_D / 10.0)); }

struct Position {
    int interval;
    double fraction, slant;
};

// npd.rs:115-150 NpdPosition::at, linear
__device__ __forceinline__ Position npd_position(const NpdLogs &L, double slant) {
    Position p;
    p.slant = fmax(slant, NPD_NEAREST_SLANT_M);
    const double lg = f_log10(p.slant / METRES_PER_FOOT);
    int interval = 0;
#pragma unroll
    for (int k = ND - 2; k >= 1; --k)
        if (interval == 0 && lg > L.lg[k]) interval = k;
    p.interval = interval;
    p.fraction = (lg - L.lg[interval]) / (L.lg[interval + 1] - L.lg[interval]);
    return p;
}

__device__ __forceinline__ double npd_linear(const Position &p, const double *curve) {
    const double lower = curve[p.interval];
    return lower + p.fraction * (curve[p.interval + 1] - lower);
}

// boxes.rs:137-149 box_level_db
// `spherical`: 20 log10 of the slant over 25,000 ft, taken once a piece.
__device__ __forceinline__ double box_level_db(const NpdLogs &L, const double *levels, double tail_db,
                                               const Position &p, double spherical) {
    const double last = levels[ND - 1];
    if (p.slant < NPD_LAST_DISTANCE_M) return npd_linear(p, levels);
    if (isinf(last) && last < 0.0) return -CUDART_INF;
    const double absorption =
        fmax((last - L.tail_anchor_db - tail_db) / (TAIL_ANCHOR_M - NPD_LAST_DISTANCE_M), 0.0);
    return last - spherical - absorption * (p.slant - NPD_LAST_DISTANCE_M);
}

// corrections.rs:33-42
__device__ __forceinline__ double finite_fraction(double along, double length, double scaled) {
    if (length < 1.0 || scaled < 1.0) return 1.0;
    const double a0 = -along / scaled, a1 = -(along - length) / scaled;
    const double e0 = a0 / (1.0 + a0 * a0) + f_atan(a0), e1 = a1 / (1.0 + a1 * a1) + f_atan(a1);
    return fmax((e1 - e0) / PI_D, 1e-15);
}

// corrections.rs:48-64
__device__ __forceinline__ double lateral_attenuation_db(double height, double lateral) {
    const double beta = f_atan(height / fmax(lateral, 0.01)) * (180.0 / PI_D);
    if (beta > 50.0) return 0.0;
    const double gamma = lateral <= 914.0 ? 1.089 * (1.0 - f_exp(-0.00274 * lateral)) : 1.0;
    const double lambda = beta < 0.0 ? 10.857 : 1.137 - 0.0229 * beta + 9.72 * f_exp(-0.142 * beta);
    return gamma * lambda;
}

// corrections.rs:69-85, wing (0) and fuselage (1); propellers take 1
__device__ __forceinline__ double installation_gain(int installation, double height, double slant) {
    const double a = installation == 0 ? 0.0039 : 0.1225;
    const double b = installation == 0 ? 0.062 : 0.329;
    const double c = installation == 0 ? 0.8786 : 1.0;
    height = fmax(height, 0.0);
    const double s2 = height * height / fmax(slant * slant, 1e-12);
    const double c2 = 1.0 - s2;
    const double num = a * c2 + s2;
    const double den = c * 4.0 * s2 * c2 + (c2 - s2) * (c2 - s2);
    return (den > 0.0 && num > 0.0) ? f_pow(num, b) / den : 1.0;
}

// popup/src/aircraft/horizons.rs:84-112 SectorEdges::loss_db over the card floats at `at`, in two
// parts. The first: no loss for a point within a metre or at or above the steepest tangent of all
// (`range` its horizontal distance).
__device__ __forceinline__ bool horizon_may_screen(const float *at, double x, double y, double z, double &range) {
    range = f_hypot(x, y);
    return !(range <= 1.0 || z >= (double)at[0] * range);
}

// The second: the point's sector, its steepest tangent, and the largest loss of its blocking edges.
__device__ __noinline__ double horizon_sector_loss_db(const float *at, int sectors, double x, double y, double z,
                                                      double range) {
    double angle = fmod(atan2(y, x), TAU_D);
    if (angle < 0.0) angle += TAU_D;
    const int sector = min((int)(angle / TAU_D * (double)sectors), sectors - 1);
    const float *e = at + 1 + sector * (1 + 2 * QM_HORIZON_BANDS);
    if (z >= (double)e[0] * range) return 0.0;
    // The largest loss of the blocking edges is the loss of their largest path difference (the loss
    // grows with it): one logarithm a lookup, and the direct path taken once.
    const double direct = f_hypot(range, z);
    double worst = 0.0;
    bool blocked = false;
#pragma unroll 1
    for (int band = 0; band < QM_HORIZON_BANDS; ++band) {
        const double r = e[1 + 2 * band], t = e[2 + 2 * band];
        if (isnan(r)) continue;
        const double eh = t * r;
        if (!(r < range && eh * range > z * r)) continue;  // screening.rs:35-38
        const double delta = f_hypot(r, eh) + f_hypot(range - r, z - eh) - direct;
        worst = blocked ? fmax(worst, delta) : delta;
        blocked = true;
    }
    if (!blocked) return 0.0;
    const double raw = 10.0 * f_log10(3.0 + PATH_DIFFERENCE_SLOPE_PER_M * fmax(worst, 0.0));
    return fmin(fmax(raw - GRAZING_LOSS_DB, 0.0), SCREENING_CAP_DB);
}

// boxes.rs:198-280 average_piece_sel: one average piece's SEL energy per period at the point before
// screening, the centroid `c` relative to it, at `gradient`; with its lateral attenuation and the two
// points its horizons are asked at (the closest point of the line for terrain, of the piece for
// buildings).
__device__ void average_piece_sel(const NpdLogs &L, const BoxDev &b, const double c[3], double gradient,
                                  double sel[3], double &lateral_out, double on_line_out[3], double on_segment_out[3]) {
    const double half = 0.5 * fmax(b.average_length, 1.0);
    const double step[3] = {b.cos_axis * half, b.sin_axis * half, gradient * half};
    double s[3], d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s[k] = c[k] - step[k];
        d[k] = (c[k] + step[k]) - s[k];
    }
    // segment.rs:223-265 closest_points, the receiver at the origin
    const double h2 = d[0] * d[0] + d[1] * d[1];
    const double l2 = h2 + d[2] * d[2];
    double along, on_line[3], on_segment[3], lateral, height, lambda_height;
    if (h2 <= 1e-6) {
        along = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) on_line[k] = on_segment[k] = s[k];
        lateral = f_hypot(s[0], s[1]);
        height = lambda_height = s[2];
    } else {
        along = -(s[0] * d[0] + s[1] * d[1] + s[2] * d[2]) / l2;
        const double clamped = fmin(fmax(along, 0.0), 1.0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            on_line[k] = s[k] + along * d[k];
            on_segment[k] = s[k] + clamped * d[k];
        }
        lateral = fabs(s[0] * d[1] - s[1] * d[0]) / sqrt(h2);
        const double slant2 = on_line[0] * on_line[0] + on_line[1] * on_line[1] + on_line[2] * on_line[2];
        height = copysign(sqrt(fmax(slant2 - lateral * lateral, 0.0)), on_line[2]);
        const double cos_climb = sqrt(h2 / l2);
        lambda_height = (along >= 0.0 && along <= 1.0) ? height : on_segment[2] / cos_climb;
    }
    const double length = fmax(sqrt(l2), 1.0);
    const double slant = f_hypot(f_hypot(on_line[0], on_line[1]), on_line[2]);
    const Position pos = npd_position(L, slant);
    const double scaled = f_exp(npd_linear(pos, b.lg_scaled) * LN10_D);
    const double along_m = along * length;
    const double stretch = f_hypot(gradient, 1.0);
    const double lateral_db = lateral_attenuation_db(lambda_height, lateral);
    const double corrections[3] = {installation_gain(0, height, slant), installation_gain(1, height, slant), 1.0};
    const double fraction = fmin(fmax(f_log10(slant / SHARE_NEAR_M) / L.lg_share_span, 0.0), 1.0);
    const double spherical = pos.slant < NPD_LAST_DISTANCE_M ? 0.0 : 20.0 * f_log10(pos.slant / NPD_LAST_DISTANCE_M);
    // The screening's gain is applied by the caller once the horizons are read (it multiplies last).
    lateral_out = lateral_db;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        on_line_out[k] = on_line[k];
        on_segment_out[k] = on_segment[k];
    }
#pragma unroll 1
    for (int p = 0; p < 3; ++p) {
        if (b.silent & (1u << p)) {
            sel[p] = 0.0;
            continue;
        }
        const double len = fmax(b.piece_length[p] * stretch, 1.0);
        const double finite = finite_fraction(along_m + 0.5 * (len - length), len, scaled);
        double parts = 0.0;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double share = b.shares[p][0][k] + fraction * (b.shares[p][1][k] - b.shares[p][0][k]);
            parts += share * corrections[k];
        }
        const double installation = parts > 0.0 ? parts : 1.0;
        sel[p] = energy_of(box_level_db(L, b.levels[p], b.tail[p], pos, spherical)) * finite * installation;
    }
}

// paint/src/flight_boxes.rs:24-33
__device__ __forceinline__ double flight_weight(uint32_t kind, double distance, double coarse) {
    if (kind == QM_FLIGHT_WEIGHT_ONE) return 1.0;
    const double f = fmin(fmax((distance - 1.5 * coarse) / (1.5 * coarse), 0.0), 1.0);
    const double far = f * f * (3.0 - 2.0 * f);
    return kind == QM_FLIGHT_WEIGHT_FAR ? far : 1.0 - far;
}

// popup/src/aircraft.rs:86-95: the class of a pass heard at `e` while `passing` of the period; the
// cast saturates as Rust's does.
__device__ __forceinline__ int pass_class(double e, double passing) {
    const double level = 10.0 * f_log10(e / passing);
    const double at = fmax((level - QM_PASS_LOWEST_DB) / QM_PASS_CLASS_DB, 0.0);
    return at >= (double)(CLASSES - 1) ? CLASSES - 1 : (int)at;
}

// Decodes the caller's boxes (DeviceFlightBoxes::upload): one thread a box.
__global__ void derive_boxes_kernel(const qm_flight_box *in, uint32_t n, BoxDev *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const qm_flight_box &a = in[i];
    BoxDev b;
    b.east = a.east_m;
    b.north = a.north_m;
    b.centroid_alt = a.centroid_altitude_m;
    b.ground = a.ground_m;
    sincos(a.axis_rad, &b.sin_axis, &b.cos_axis);
    b.gradient = a.gradient;
    b.spread = a.gradient_spread;
    b.pad0 = 0.0;
    // boxes.rs:93-107 average_length_m: the periods' lengths weighed by their energy at 1,000 ft
    double w[3], total = 0.0;
#pragma unroll
    for (int p = 0; p < 3; ++p) total += (w[p] = energy_of(a.levels_db[p][3]));
    if (total > 0.0) {
        double sum = 0.0;
#pragma unroll
        for (int p = 0; p < 3; ++p) sum += w[p] * a.piece_length_m[p];
        b.average_length = sum / total;
    } else {
        b.average_length = a.piece_length_m[0];
    }
    uint32_t silent = 0;
    for (int p = 0; p < 3; ++p) {
        b.piece_length[p] = a.piece_length_m[p];
        b.passing[p] = a.passing[p];
        b.tail[p] = a.tail_levels_db[p];
        bool all = true;
        for (int k = 0; k < ND; ++k) {
            b.levels[p][k] = a.levels_db[p][k];
            all = all && isinf(a.levels_db[p][k]) && a.levels_db[p][k] < 0.0;
        }
        if (all) silent |= 1u << p;
        for (int s = 0; s < 2; ++s)
            for (int k = 0; k < 3; ++k) b.shares[p][s][k] = a.installation_shares[p][s][k];
    }
    for (int k = 0; k < ND; ++k) b.lg_scaled[k] = a.lg_scaled_distance[k];
    b.helicopter = a.helicopter;
    b.silent = silent;
    out[i] = b;
}

// One CTA's share of a request band: reads [read_begin, read_end) of the ordered segments
// [seg_begin, seg_end) (positions in `order`), all adding to sums `sum`; `point` >= 0 when every
// one of those segments names that point (its horizons are then staged in shared memory).
struct Slice {
    uint64_t read_begin, read_end;
    uint32_t seg_begin, seg_end;
    uint32_t sum;
    int32_t point;
};

struct SumsArgs {
    const BoxDev *boxes;
    const qm_flight_point *points;
    const float *horizons;  // nullable: free field
    const qm_box_segment *segments;
    const uint32_t *order;        // segment indices grouped by sum, each group in the caller's order
    const uint64_t *read_start;   // per ordered position: the reads of the positions before it
    const Slice *slices;
    double *sums;                 // [n_sums][QM_FLIGHT_SUMS], zeroed
    unsigned long long *heard;    // boxes within reach with a positive weight
    NpdLogs logs;
};

constexpr int WARPS = THREADS / 32;

// A heard box waiting in its warp's queue: the box, its ordered segment position and its weight.
struct Heard {
    uint32_t box, at;
    double share;
};

// The point of ordered segment position `at`, and its horizons: the slice's staged copy when the
// slice stages that point's, else the caller's floats (nullptr: free field).
struct PointView {
    qm_flight_point pt;
    const float *horizons;
};

__device__ __forceinline__ PointView point_of(const SumsArgs &A, const Slice &sl, const float *staged, uint32_t at) {
    const uint32_t point = A.segments[A.order[at]].point;
    PointView v;
    v.pt = A.points[point];
    v.horizons = (int32_t)point == sl.point ? staged : (A.horizons ? A.horizons + v.pt.horizons : nullptr);
    return v;
}

// A warp's working space for up to 32 boxes' average pieces (two a box at most).
struct WarpWork {
    double sel[64][3];      // each piece's SEL energy per period before screening
    double lateral[64];     // its lateral attenuation (dB)
    double loss[64][2];     // its terrain and building losses (dB)
    // A round's horizon lookups that passed their first test: per lane of the round its piece, its
    // point's horizons and the two points with their ranges; the queue holds 2 x lane + horizon.
    double point[32][2][4];
    const float *horizons[32];
    int piece[32];
    int look[64];
};

// The first `n` (at most 32) boxes of a warp's queue: their average pieces (one a box, two for a
// box whose gradients spread) spread over the lanes, one piece a lane; the horizon lookups that
// pass their first test queued and read on full warps; then each box's pieces joined by its own lane
// with their screening gains into period energies and pass classes (popup/src/aircraft/boxes.rs:
// 187-223 box_at, popup/src/aircraft.rs:86-95 add_pass).
__device__ void evaluate_queue(const SumsArgs &A, const Slice &sl, const float *staged, const Heard *queue,
                               WarpWork &w, int n, int lane, double energy[3], double *class_energy,
                               double *class_passing) {
    bool two = false;
    if (lane < n) two = A.boxes[queue[lane].box].spread > 0.0;
    const unsigned twos = __ballot_sync(0xffffffffu, two);
    const int total = n + __popc(twos);
    const unsigned below = (1u << lane) - 1u;
    for (int k0 = 0; k0 < total; k0 += 32) {
        const int k = k0 + lane;
        bool t_look = false, b_look = false;
        if (k < total) {
            const int slot = k < n ? k : (int)__fns(twos, 0, k - n + 1);
            const int which = k < n ? 0 : 1;
            const int piece = 2 * slot + which;
            const Heard h = queue[slot];
            const BoxDev &b = A.boxes[h.box];
            const PointView v = point_of(A, sl, staged, h.at);
            const double c[3] = {b.east - v.pt.x, b.north - v.pt.y, b.centroid_alt - v.pt.altitude_m};
            const bool screened = c[2] - (b.ground - v.pt.altitude_m) < SCREENING_CEILING_M;
            const double spread = b.spread;
            const double gradient = spread > 0.0 ? (which ? b.gradient + spread : b.gradient - spread) : b.gradient;
            double on_line[3], on_segment[3];
            average_piece_sel(A.logs, b, c, gradient, w.sel[piece], w.lateral[piece], on_line, on_segment);
            w.loss[piece][0] = w.loss[piece][1] = 0.0;
            if (screened && v.horizons) {
                double r;
                w.piece[lane] = piece;
                w.horizons[lane] = v.horizons;
                if (horizon_may_screen(v.horizons, on_line[0], on_line[1], on_line[2], r)) {
                    t_look = true;
                    w.point[lane][0][0] = on_line[0];
                    w.point[lane][0][1] = on_line[1];
                    w.point[lane][0][2] = on_line[2];
                    w.point[lane][0][3] = r;
                }
                if (horizon_may_screen(v.horizons + QM_TERRAIN_HORIZON_FLOATS, on_segment[0], on_segment[1],
                                       on_segment[2], r)) {
                    b_look = true;
                    w.point[lane][1][0] = on_segment[0];
                    w.point[lane][1][1] = on_segment[1];
                    w.point[lane][1][2] = on_segment[2];
                    w.point[lane][1][3] = r;
                }
            }
        }
        const unsigned mt = __ballot_sync(0xffffffffu, t_look), mb = __ballot_sync(0xffffffffu, b_look);
        if (t_look) w.look[__popc(mt & below)] = 2 * lane;
        if (b_look) w.look[__popc(mt) + __popc(mb & below)] = 2 * lane + 1;
        const int n_look = __popc(mt) + __popc(mb);
        __syncwarp();
        for (int j = lane; j < n_look; j += 32) {
            const int src = w.look[j] >> 1, hz = w.look[j] & 1;
            const double *q = w.point[src][hz];
            const float *at = w.horizons[src] + (hz ? QM_TERRAIN_HORIZON_FLOATS : 0);
            w.loss[w.piece[src]][hz] =
                horizon_sector_loss_db(at, hz ? QM_BUILDING_SECTORS : QM_TERRAIN_SECTORS, q[0], q[1], q[2], q[3]);
        }
        __syncwarp();
    }
    if (lane < n) {
        const Heard h = queue[lane];
        const BoxDev &b = A.boxes[h.box];
        const double impedance = b.helicopter ? 1.0 : A.points[A.segments[A.order[h.at]].point].impedance_gain;
        // screening.rs:48-55 screened_sel_db(0, ...) less the lateral attenuation, a piece's gain
        auto gain_of = [&](int piece) {
            const double lat = w.lateral[piece];
            return energy_of((0.0 - fmax(fmax(w.loss[piece][0], w.loss[piece][1]) - lat, 0.0)) - lat);
        };
        const double g0 = gain_of(2 * lane), g1 = two ? gain_of(2 * lane + 1) : 0.0;
#pragma unroll 1
        for (int p = 0; p < 3; ++p) {
            const double lo = w.sel[2 * lane][p] * g0;
            const double s = two ? 0.5 * (lo + w.sel[2 * lane + 1][p] * g1) : lo;
            const double hours = p == 0 ? 12.0 : p == 1 ? 4.0 : 8.0;  // physics/src/bands.rs:16
            const double e = h.share * (s * impedance / (hours * 3600.0));
            const double passing = h.share * b.passing[p];
            energy[p] += e;
            if (e > 0.0 && passing > 0.0) {
                const int k = p * CLASSES + pass_class(e, passing);
                atomicAdd(&class_energy[k], e);
                atomicAdd(&class_passing[k], passing);
            }
        }
    }
    __syncwarp();
}

// One CTA a slice of one request band's reads. Each warp tests 32 reads at a time against the
// reach and the lattice weight (paint/src/flight_boxes.rs:24-33), queues the heard ones and
// evaluates its queue 32 boxes at a time, so that the equation runs on full warps.
__global__ void __launch_bounds__(THREADS) flight_sums_kernel(SumsArgs A) {
    __shared__ float s_horizons[QM_HORIZON_FLOATS];
    __shared__ double s_class_energy[3 * CLASSES], s_class_passing[3 * CLASSES];
    __shared__ double s_energy[3][THREADS];
    __shared__ Heard s_queue[WARPS][64];
    __shared__ WarpWork s_work[WARPS];
    __shared__ unsigned s_heard;
    const Slice sl = A.slices[blockIdx.x];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int k = tid; k < 3 * CLASSES; k += THREADS) s_class_energy[k] = s_class_passing[k] = 0.0;
    if (tid == 0) s_heard = 0;
    const float *staged = nullptr;
    if (sl.point >= 0 && A.horizons) {
        const float *src = A.horizons + A.points[sl.point].horizons;
        for (int k = tid; k < QM_HORIZON_FLOATS; k += THREADS) s_horizons[k] = __ldg(src + k);
        staged = s_horizons;
    }
    __syncthreads();
    double energy[3] = {0.0, 0.0, 0.0};
    unsigned heard = 0;
    int queued = 0;  // warp-uniform
    Heard *queue = s_queue[warp];
    for (uint64_t base = sl.read_begin + (uint64_t)warp * 32; base < sl.read_end; base += THREADS) {
        const uint64_t r = base + lane;
        bool hit = false;
        Heard h;
        if (r < sl.read_end) {
            // The ordered segment holding read r: the last position whose start is at most r.
            uint32_t lo = sl.seg_begin, hi = sl.seg_end - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (A.read_start[mid] <= r) lo = mid;
                else hi = mid - 1;
            }
            const qm_box_segment seg = A.segments[A.order[lo]];
            const qm_flight_point &pt = A.points[seg.point];
            const uint32_t box = seg.first + (uint32_t)(r - A.read_start[lo]);
            const double distance = f_hypot(__ldg(&A.boxes[box].east) - pt.x, __ldg(&A.boxes[box].north) - pt.y);
            const double reach = fmin(seg.within_m, QM_AIRCRAFT_REACH_M);
            const double share = distance <= reach ? flight_weight(seg.weight, distance, seg.coarse_m) : 0.0;
            hit = share > 0.0;
            h.box = box;
            h.at = lo;
            h.share = share;
        }
        const unsigned mask = __ballot_sync(0xffffffffu, hit);
        if (hit) queue[queued + __popc(mask & ((1u << lane) - 1u))] = h;
        queued += __popc(mask);
        heard += hit ? 1u : 0u;
        __syncwarp();
        if (queued >= 32) {
            evaluate_queue(A, sl, staged, queue, s_work[warp], 32, lane, energy, s_class_energy, s_class_passing);
            const bool move = lane < queued - 32;
            Heard keep;
            if (move) keep = queue[32 + lane];
            __syncwarp();
            if (move) queue[lane] = keep;
            __syncwarp();
            queued -= 32;
        }
    }
    if (queued > 0)
        evaluate_queue(A, sl, staged, queue, s_work[warp], queued, lane, energy, s_class_energy, s_class_passing);
#pragma unroll
    for (int p = 0; p < 3; ++p) s_energy[p][tid] = energy[p];
    if (heard) atomicAdd(&s_heard, heard);
    __syncthreads();
    double *out = A.sums + (size_t)sl.sum * QM_FLIGHT_SUMS;
    if (tid < 3) {
        double total = 0.0;
        for (int t = 0; t < THREADS; ++t) total += s_energy[tid][t];
        if (total != 0.0) atomicAdd(&out[tid], total);
    }
    for (int k = tid; k < 3 * CLASSES; k += THREADS) {
        if (s_class_energy[k] != 0.0) atomicAdd(&out[3 + k], s_class_energy[k]);
        if (s_class_passing[k] != 0.0) atomicAdd(&out[3 + 3 * CLASSES + k], s_class_passing[k]);
    }
    if (tid == 0 && s_heard) atomicAdd(A.heard, (unsigned long long)s_heard);
}

}  // namespace fl
}  // namespace qm
