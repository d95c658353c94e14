// FP64 CPU oracle of the Doc 29 aircraft path — TEST INFRASTRUCTURE ONLY.
//
// Restates the reference's segment SEL at a receiver (physics/src/doc29/segment.rs:223-345), its NPD
// reading (physics/src/doc29/npd.rs:115-277) and corrections (physics/src/doc29/corrections.rs:21-85)
// in double precision, and sums segments over a receiver grid into third-octave spectra whose
// Zwicker loudness (physics/src/loudness.rs, restated in qm_oracle.cpp) is the cell's sone.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../include/qm_aircraft.h"
#include "../include/qm_flights.h"

extern "C" double qmo_zwicker(const double *levels28);

namespace {

constexpr int ND = 10;
constexpr double METRES_PER_FOOT = 0.3048;
const double NPD_DISTANCES_FT[ND] = {200.0, 400.0, 630.0, 1000.0, 2000.0, 4000.0, 6300.0, 10000.0, 16000.0, 25000.0};
constexpr double NPD_NEAREST_SLANT_M = 100.0 * METRES_PER_FOOT;
constexpr double NPD_LAST_DISTANCE_M = 25000.0 * METRES_PER_FOOT;
constexpr double PI = 3.141592653589793116;
constexpr double LN10 = 2.302585092994045684;
// Third-octave A-weighting, 25 Hz .. 12.5 kHz (physics/src/loudness.rs:14-17).
const double A_WEIGHTING_THIRDS[28] = {-44.7, -39.4, -34.6, -30.2, -26.2, -22.5, -19.1, -16.1, -13.4, -10.9,
                                       -8.6,  -6.6,  -4.8,  -3.2,  -1.9,  -0.8,  0.0,   0.6,   1.0,   1.2,
                                       1.3,   1.2,   1.0,   0.5,   -0.1,  -1.1,  -2.5,  -4.3};

inline double energy(double level_db) { return std::exp(level_db * (LN10 / 10.0)); }

// npd.rs:115-150
struct NpdPosition {
    int interval;
    double fraction, slant_m;
    static NpdPosition at(double slant_m) {
        slant_m = std::max(slant_m, NPD_NEAREST_SLANT_M);
        double log_d = std::log10(slant_m / METRES_PER_FOOT);
        int interval = 0;
        for (int k = ND - 2; k >= 1; --k)
            if (log_d > std::log10(NPD_DISTANCES_FT[k])) {
                interval = k;
                break;
            }
        double l0 = std::log10(NPD_DISTANCES_FT[interval]), l1 = std::log10(NPD_DISTANCES_FT[interval + 1]);
        return NpdPosition{interval, (log_d - l0) / (l1 - l0), slant_m};
    }
    double linear(const double *curve) const {
        double lower = curve[interval];
        return lower + fraction * (curve[interval + 1] - lower);
    }
    // npd.rs:155-163
    double level(const double *curve, double tail_absorption_db_per_m) const {
        if (slant_m < NPD_LAST_DISTANCE_M) return linear(curve);
        return curve[ND - 1] - 20.0 * std::log10(slant_m / NPD_LAST_DISTANCE_M) -
               tail_absorption_db_per_m * (slant_m - NPD_LAST_DISTANCE_M);
    }
};

// npd.rs:169-186
double tail_absorption_db_per_m(const double *sel) {
    double sx = 0, sy = 0, sxx = 0, sxy = 0;
    for (int i = 0; i < 3; ++i) {
        int k = ND - 3 + i;
        double d = NPD_DISTANCES_FT[k] * METRES_PER_FOOT;
        double y = sel[k] + 20.0 * std::log10(d / NPD_LAST_DISTANCE_M);
        sx += d;
        sy += y;
        sxx += d * d;
        sxy += d * y;
    }
    double n = 3.0;
    return std::max(-(n * sxy - sx * sy) / (n * sxx - sx * sx), 0.0);
}

struct NpdReading {
    double sel_db, lamax_db, scaled_distance_m;
};

// npd.rs:238-277 PowerRow (an event-duration row: SEL - LAmax is no 12 dB placeholder here)
struct PowerRow {
    double sel[ND], lamax[ND], sel_minus_lamax[ND];
    double tail_alpha, d0_m;
    bool dipole;
    NpdReading read(const NpdPosition &p) const {
        double scaled = dipole ? p.slant_m : d0_m * energy(p.linear(sel_minus_lamax));
        return NpdReading{p.level(sel, tail_alpha), p.level(lamax, tail_alpha), scaled};
    }
};

PowerRow make_row(const float *sel, const float *lamax, double v_ref_kt) {
    PowerRow r;
    bool placeholder = true;
    for (int k = 0; k < ND; ++k) {
        r.sel[k] = sel[k];
        r.lamax[k] = lamax[k];
        r.sel_minus_lamax[k] = r.sel[k] - r.lamax[k];
        if (std::fabs(r.sel_minus_lamax[k] - 12.0) >= 1e-9) placeholder = false;
    }
    r.dipole = placeholder;
    double speed = v_ref_kt * 1852.0 / 3600.0;
    r.d0_m = 2.0 / PI * speed * 1.0;
    r.tail_alpha = tail_absorption_db_per_m(r.sel);
    return r;
}

// corrections.rs:21-27
double speed_correction_db(double v_ref_kt, double speed_kt) {
    return speed_kt > 10.0 ? 10.0 * std::log10(v_ref_kt / speed_kt) : 0.0;
}

// corrections.rs:33-42
double finite_segment_energy_fraction(double along_m, double length_m, double scaled_m) {
    if (length_m < 1.0 || scaled_m < 1.0) return 1.0;
    double a0 = -along_m / scaled_m, a1 = -(along_m - length_m) / scaled_m;
    auto e = [](double a) { return a / (1.0 + a * a) + std::atan(a); };
    return std::max((e(a1) - e(a0)) / PI, 1e-15);
}

// corrections.rs:48-64
double lateral_attenuation_db(double height_m, double lateral_m) {
    double beta = std::atan(height_m / std::max(lateral_m, 0.01)) * (180.0 / PI);
    if (beta > 50.0) return 0.0;
    double gamma = lateral_m <= 914.0 ? 1.089 * (1.0 - std::exp(-0.00274 * lateral_m)) : 1.0;
    double lambda = beta < 0.0 ? 10.857 : 1.137 - 0.0229 * beta + 9.72 * std::exp(-0.142 * beta);
    return gamma * lambda;
}

// corrections.rs:69-85
double installation_energy_gain(uint32_t installation, double height_m, double slant_m) {
    double a, b, c;
    if (installation == 0) {
        a = 0.0039;
        b = 0.062;
        c = 0.8786;
    } else if (installation == 1) {
        a = 0.1225;
        b = 0.329;
        c = 1.0;
    } else {
        return 1.0;
    }
    height_m = std::max(height_m, 0.0);
    double s2 = height_m * height_m / std::max(slant_m * slant_m, 1e-12);
    double c2 = 1.0 - s2;
    double num = a * c2 + s2;
    double den = c * 4.0 * s2 * c2 + (c2 - s2) * (c2 - s2);
    return (den > 0.0 && num > 0.0) ? std::pow(num, b) / den : 1.0;
}

struct Closest {
    double along, on_line[3], on_segment[3], lateral, height, lambda_height, length;
};

// segment.rs:223-265 (the receiver at the origin)
Closest closest_points(const double s[3], const double e[3]) {
    double d[3] = {e[0] - s[0], e[1] - s[1], e[2] - s[2]};
    double h2 = d[0] * d[0] + d[1] * d[1];
    double l2 = h2 + d[2] * d[2];
    Closest c;
    if (h2 <= 1e-6) {
        c.along = 0.0;
        for (int k = 0; k < 3; ++k) c.on_line[k] = c.on_segment[k] = s[k];
        c.lateral = std::hypot(s[0], s[1]);
        c.height = s[2];
        c.lambda_height = s[2];
        c.length = std::max(std::sqrt(l2), 1.0);
        return c;
    }
    double along = -(s[0] * d[0] + s[1] * d[1] + s[2] * d[2]) / l2;
    double clamped = std::min(std::max(along, 0.0), 1.0);
    for (int k = 0; k < 3; ++k) {
        c.on_line[k] = s[k] + along * d[k];
        c.on_segment[k] = s[k] + clamped * d[k];
    }
    c.along = along;
    c.lateral = std::fabs(s[0] * d[1] - s[1] * d[0]) / std::sqrt(h2);
    double slant2 = c.on_line[0] * c.on_line[0] + c.on_line[1] * c.on_line[1] + c.on_line[2] * c.on_line[2];
    c.height = std::copysign(std::sqrt(std::max(slant2 - c.lateral * c.lateral, 0.0)), c.on_line[2]);
    double cos_climb = std::sqrt(h2 / l2);
    c.lambda_height = (along >= 0.0 && along <= 1.0) ? c.height : c.on_segment[2] / cos_climb;
    c.length = std::max(std::sqrt(l2), 1.0);
    return c;
}

struct Type {
    PowerRow rows[2][10];
    double v_ref_kt;
    uint32_t installation;
    double share[28];  // unweighted band energy per unit A-weighted energy
};

Type make_type(const qm_aircraft_type &a) {
    Type T;
    T.v_ref_kt = a.v_ref_kt;
    T.installation = a.installation;
    for (int op = 0; op < 2; ++op)
        for (int r = 0; r < 10; ++r) T.rows[op][r] = make_row(a.sel_db[op][r], a.lamax_db[op][r], a.v_ref_kt);
    double weighted = 0.0;
    for (int b = 0; b < 28; ++b) weighted += energy(a.spectrum_db[b] + A_WEIGHTING_THIRDS[b]);
    for (int b = 0; b < 28; ++b) T.share[b] = energy(a.spectrum_db[b]) / weighted;
    return T;
}

// screened_segment_sel (segment.rs:317-345) with no horizons, read_npd's power lerp (npd.rs:189-203)
double segment_sel_db(const Type &T, const qm_flight_segment &g, double rx, double ry, double rz) {
    double s[3] = {g.start[0] - rx, g.start[1] - ry, g.start[2] - rz};
    double e[3] = {g.end[0] - rx, g.end[1] - ry, g.end[2] - rz};
    Closest c = closest_points(s, e);
    double slant = std::sqrt(c.on_line[0] * c.on_line[0] + c.on_line[1] * c.on_line[1] + c.on_line[2] * c.on_line[2]);
    NpdPosition pos = NpdPosition::at(slant);
    int row = std::min((int)std::floor(g.power), 8);
    double weight = g.power - row;
    const PowerRow *rows = T.rows[g.departure ? 1 : 0];
    NpdReading low = rows[row].read(pos);
    NpdReading npd = low;
    if (weight != 0.0) {
        NpdReading high = rows[row + 1].read(pos);
        npd.sel_db = low.sel_db + weight * (high.sel_db - low.sel_db);
        npd.lamax_db = low.lamax_db + weight * (high.lamax_db - low.lamax_db);
        npd.scaled_distance_m = low.scaled_distance_m + weight * (high.scaled_distance_m - low.scaled_distance_m);
    }
    double speed_kt = g.speed_mps * 3600.0 / 1852.0;
    double finite = 10.0 * std::log10(finite_segment_energy_fraction(c.along * c.length, c.length, npd.scaled_distance_m));
    double lateral = lateral_attenuation_db(c.lambda_height, c.lateral);
    double installation = 10.0 * std::log10(installation_energy_gain(T.installation, c.height, slant));
    return npd.sel_db + speed_correction_db(T.v_ref_kt, speed_kt) + installation - lateral + finite;
}

// ---- Aircraft boxes: the builder's sums and the click-time equation -------------------------

constexpr double TAIL_ANCHOR_M = 16000.0;                             // npd.rs:330
const double INSTALLATION_SHARE_SLANTS_M[2] = {1000.0 * METRES_PER_FOOT, TAIL_ANCHOR_M};  // box_sums.rs:14
constexpr int GEOMETRY_DISTANCE = 3;                                  // box_sums.rs:11, boxes.rs:30
constexpr double PATH_DIFFERENCE_SLOPE_PER_M = 29.2;                  // screening.rs:8
constexpr double GRAZING_LOSS_DB = 4.771212547196624;                 // screening.rs:10
constexpr double SCREENING_CAP_DB = 18.0;                             // screening.rs:12
constexpr double SCREENING_CEILING_ABOVE_GROUND_M = 7620.0;           // screening.rs:15
constexpr double AIRCRAFT_REACH_M = 16000.0;                          // popup/src/aircraft/boxes.rs:22
const double PERIOD_HOURS_D[3] = {12.0, 4.0, 8.0};                    // bands.rs:16
constexpr int PASS_CLASSES = 48;                                      // popup/src/aircraft.rs:51-53
constexpr double PASS_CLASS_DB = 3.0, PASS_LOWEST_DB = -30.0;
constexpr int HORIZON_BANDS = 6;

inline double level_of(double e) { return e > 0.0 ? 10.0 * std::log10(e) : -INFINITY; }

// A segment's energies at the NPD distances and the tail anchor (box_sums.rs:17-33 with the
// segment's NpdDistanceLevels, segment.rs:172-180): the power-lerped reading plus Delta_V.
struct SegmentEnergies {
    double unweighted[ND], tail, scaled_distance_m[ND];
};

NpdReading read_npd(const Type &T, const qm_flight_segment &g, double slant_m) {
    NpdPosition pos = NpdPosition::at(slant_m);
    int row = std::min((int)std::floor(g.power), 8);
    double weight = g.power - row;
    const PowerRow *rows = T.rows[g.departure ? 1 : 0];
    NpdReading low = rows[row].read(pos);
    if (weight == 0.0) return low;
    NpdReading high = rows[row + 1].read(pos);
    return NpdReading{low.sel_db + weight * (high.sel_db - low.sel_db),
                      low.lamax_db + weight * (high.lamax_db - low.lamax_db),
                      low.scaled_distance_m + weight * (high.scaled_distance_m - low.scaled_distance_m)};
}

SegmentEnergies segment_energies(const Type &T, const qm_flight_segment &g) {
    double dv = speed_correction_db(T.v_ref_kt, g.speed_mps * 3600.0 / 1852.0);
    SegmentEnergies s;
    for (int k = 0; k < ND; ++k) {
        NpdReading r = read_npd(T, g, NPD_DISTANCES_FT[k] * METRES_PER_FOOT);
        s.unweighted[k] = std::pow(10.0, (r.sel_db + dv) / 10.0);
        s.scaled_distance_m[k] = r.scaled_distance_m;
    }
    s.tail = std::pow(10.0, (read_npd(T, g, TAIL_ANCHOR_M).sel_db + dv) / 10.0);
    return s;
}

// The running sums of one box (box_sums.rs:35-60, add :82-142).
struct BoxSums {
    double energy[3][ND] = {}, tail_energy[3] = {}, energy_over_scaled_distance[ND] = {};
    double weight = 0.0, weighted_midpoint_m[3] = {};
    double period_weight[3] = {}, period_weighted_length_m[3] = {};
    double weighted_doubled_direction[2] = {}, weighted_gradient_direction[2] = {}, weighted_squared_gradient[3] = {};
    double installation_energy[3][2][3] = {};

    void add(const SegmentEnergies &en, uint32_t installation, const double period_weights[3], const double start[3],
             const double end[3]) {
        double total_weight = period_weights[0] + period_weights[1] + period_weights[2];
        if (total_weight <= 0.0) return;
        for (int p = 0; p < 3; ++p) {
            for (int k = 0; k < ND; ++k) energy[p][k] += period_weights[p] * en.unweighted[k];
            tail_energy[p] += period_weights[p] * en.tail;
        }
        for (int k = 0; k < ND; ++k)
            energy_over_scaled_distance[k] += total_weight * en.unweighted[k] / std::max(en.scaled_distance_m[k], 1.0);
        double w = total_weight * en.unweighted[GEOMETRY_DISTANCE];
        double d[3] = {end[0] - start[0], end[1] - start[1], end[2] - start[2]};
        double length = std::hypot(d[0], d[1]);
        weight += w;
        for (int a = 0; a < 3; ++a) weighted_midpoint_m[a] += w * 0.5 * (start[a] + end[a]);
        for (int p = 0; p < 3; ++p) {
            double pw = period_weights[p] * en.unweighted[GEOMETRY_DISTANCE];
            period_weight[p] += pw;
            period_weighted_length_m[p] += pw * length;
        }
        if (length > 0.0) {
            double c = d[0] / length, s = d[1] / length;
            weighted_doubled_direction[0] += w * (c * c - s * s);
            weighted_doubled_direction[1] += w * 2.0 * s * c;
            double gradient = d[2] / length;
            weighted_gradient_direction[0] += w * gradient * c;
            weighted_gradient_direction[1] += w * gradient * s;
            double sq = w * gradient * gradient;
            weighted_squared_gradient[0] += sq * c * c;
            weighted_squared_gradient[1] += sq * s * s;
            weighted_squared_gradient[2] += sq * s * c;
        }
        uint32_t slot = installation < 2 ? installation : 2;
        for (int p = 0; p < 3; ++p) {
            installation_energy[p][0][slot] += period_weights[p] * en.unweighted[GEOMETRY_DISTANCE];
            installation_energy[p][1][slot] += period_weights[p] * en.tail;
        }
    }

    // box_sums.rs:144-199, into a box record (lg d_lambda as the tile keeps it).
    bool values(qm_flight_box &b) const {
        if (weight <= 0.0) return false;
        for (int p = 0; p < 3; ++p) {
            for (int k = 0; k < ND; ++k) b.levels_db[p][k] = level_of(energy[p][k]);
            b.tail_levels_db[p] = level_of(tail_energy[p]);
        }
        for (int k = 0; k < ND; ++k) {
            double e = energy[0][k] + energy[1][k] + energy[2][k];
            b.lg_scaled_distance[k] = std::log10(e / energy_over_scaled_distance[k]);
        }
        double axis = std::fmod(0.5 * std::atan2(weighted_doubled_direction[1], weighted_doubled_direction[0]), PI);
        if (axis < 0.0) axis += PI;
        double s = std::sin(axis), c = std::cos(axis);
        double gradient = (weighted_gradient_direction[0] * c + weighted_gradient_direction[1] * s) / weight;
        double mean_square = (weighted_squared_gradient[0] * c * c + weighted_squared_gradient[1] * s * s +
                              2.0 * weighted_squared_gradient[2] * s * c) / weight;
        b.east_m = weighted_midpoint_m[0] / weight;
        b.north_m = weighted_midpoint_m[1] / weight;
        b.centroid_altitude_m = weighted_midpoint_m[2] / weight;
        b.axis_rad = axis;
        b.gradient = gradient;
        b.gradient_spread = std::sqrt(std::max(mean_square - gradient * gradient, 0.0));
        for (int p = 0; p < 3; ++p) {
            b.piece_length_m[p] = period_weight[p] > 0.0 ? period_weighted_length_m[p] / period_weight[p] : 0.0;
            for (int slant = 0; slant < 2; ++slant) {
                const double *e = installation_energy[p][slant];
                double total = e[0] + e[1] + e[2];
                for (int k = 0; k < 3; ++k)
                    b.installation_shares[p][slant][k] = total > 0.0 ? e[k] / total : (k == 2 ? 1.0 : 0.0);
            }
        }
        return true;
    }
};

// screening.rs:19-23, 29-44, 48-55
double path_difference_loss_db(double delta) {
    double raw = 10.0 * std::log10(3.0 + PATH_DIFFERENCE_SLOPE_PER_M * std::max(delta, 0.0));
    return std::min(std::max(raw - GRAZING_LOSS_DB, 0.0), SCREENING_CAP_DB);
}

double edge_loss_db(double edge_range, double edge_height, double source_range, double source_height) {
    bool blocks = edge_range < source_range && edge_height * source_range > source_height * edge_range;
    if (!blocks) return 0.0;
    double re = std::hypot(edge_range, edge_height);
    double es = std::hypot(source_range - edge_range, source_height - edge_height);
    double rs = std::hypot(source_range, source_height);
    return path_difference_loss_db(re + es - rs);
}

double screened_sel_db(double free_db, double lateral_db, double terrain_db, double building_db) {
    return free_db - std::max(std::max(terrain_db, building_db) - lateral_db, 0.0);
}

// One horizon as the card stores it (horizons.rs:50-64 write_f32), read in double: the steepest
// tangent of all, then per sector its steepest and per band (range, tangent), NaN range empty.
struct SectorEdges {
    const float *at = nullptr;
    int sectors = 0;
    // horizons.rs:84-106 loss_db and :109-112 sector_of
    double loss_db(const double p[3]) const {
        if (!at) return 0.0;
        double range = std::hypot(p[0], p[1]);
        if (range <= 1.0 || p[2] >= (double)at[0] * range) return 0.0;
        double angle = std::fmod(std::atan2(p[1], p[0]), 2.0 * PI);
        if (angle < 0.0) angle += 2.0 * PI;
        int sector = std::min((int)(angle / (2.0 * PI) * (double)sectors), sectors - 1);
        const float *e = at + 1 + sector * (1 + 2 * HORIZON_BANDS);
        if (p[2] >= (double)e[0] * range) return 0.0;
        double loss = 0.0;
        for (int band = 0; band < HORIZON_BANDS; ++band) {
            double r = e[1 + 2 * band], t = e[2 + 2 * band];
            if (std::isnan(r)) continue;
            loss = std::max(loss, edge_loss_db(r, t * r, range, p[2]));
        }
        return loss;
    }
};

struct Horizons {
    SectorEdges terrain, buildings;
    static Horizons of(const float *floats) {
        Horizons h;
        if (floats) {
            h.terrain = SectorEdges{floats, QM_TERRAIN_SECTORS};
            h.buildings = SectorEdges{floats + QM_TERRAIN_HORIZON_FLOATS, QM_BUILDING_SECTORS};
        }
        return h;
    }
};

// A box in the receiver's frame (boxes.rs:33-56 AircraftBoxAtReceiver).
struct BoxAtReceiver {
    double centroid[3], axis, gradient, spread, ground_m;
    const qm_flight_box *b;
};

struct BoxSel {
    double sel_energy[3], fractions[3][3];
};

// boxes.rs:93-107
double average_length_m(const qm_flight_box &b) {
    double w[3], total = 0.0;
    for (int p = 0; p < 3; ++p) total += (w[p] = energy(b.levels_db[p][GEOMETRY_DISTANCE]));
    if (!(total > 0.0)) return b.piece_length_m[0];
    double sum = 0.0;
    for (int p = 0; p < 3; ++p) sum += w[p] * b.piece_length_m[p];
    return sum / total;
}

// boxes.rs:137-149
double box_level_db(const double *levels, double tail_db, const NpdPosition &pos) {
    double last = levels[ND - 1], slant = pos.slant_m;
    if (slant < NPD_LAST_DISTANCE_M) return pos.linear(levels);
    if (last == -INFINITY) return -INFINITY;
    auto spherical = [](double d) { return 20.0 * std::log10(d / NPD_LAST_DISTANCE_M); };
    double absorption = std::max((last - spherical(TAIL_ANCHOR_M) - tail_db) / (TAIL_ANCHOR_M - NPD_LAST_DISTANCE_M), 0.0);
    return last - spherical(slant) - absorption * (slant - NPD_LAST_DISTANCE_M);
}

// boxes.rs:198-280
BoxSel average_piece_sel(const BoxAtReceiver &a, const Horizons &h, double length_m) {
    const qm_flight_box &b = *a.b;
    double half = 0.5 * std::max(length_m, 1.0);
    double sn = std::sin(a.axis), cs = std::cos(a.axis);
    double step[3] = {cs * half, sn * half, a.gradient * half};
    double start[3], end[3];
    for (int k = 0; k < 3; ++k) {
        start[k] = a.centroid[k] - step[k];
        end[k] = a.centroid[k] + step[k];
    }
    Closest c = closest_points(start, end);
    double slant = std::hypot(std::hypot(c.on_line[0], c.on_line[1]), c.on_line[2]);
    NpdPosition pos = NpdPosition::at(slant);
    double scaled = std::exp(pos.linear(b.lg_scaled_distance) * LN10);
    double along = c.along * c.length;
    double stretch = std::hypot(a.gradient, 1.0);
    double lateral = lateral_attenuation_db(c.lambda_height, c.lateral);
    double corrections[3] = {installation_energy_gain(0, c.height, slant), installation_energy_gain(1, c.height, slant),
                             installation_energy_gain(2, c.height, slant)};
    double near = INSTALLATION_SHARE_SLANTS_M[0], far = INSTALLATION_SHARE_SLANTS_M[1];
    double fraction = std::min(std::max(std::log10(slant / near) / std::log10(far / near), 0.0), 1.0);
    BoxSel out;
    double installation[3];
    for (int p = 0; p < 3; ++p) {
        double shares[3], parts[3], sum = 0.0;
        for (int k = 0; k < 3; ++k) {
            shares[k] = b.installation_shares[p][0][k] + fraction * (b.installation_shares[p][1][k] - b.installation_shares[p][0][k]);
            parts[k] = shares[k] * corrections[k];
        }
        sum = parts[0] + parts[1] + parts[2];
        if (sum > 0.0) {
            installation[p] = sum;
            for (int k = 0; k < 3; ++k) out.fractions[p][k] = parts[k] / sum;
        } else {
            installation[p] = 1.0;
            for (int k = 0; k < 3; ++k) out.fractions[p][k] = shares[k];
        }
    }
    double terrain = 0.0, building = 0.0;
    if (a.centroid[2] - a.ground_m < SCREENING_CEILING_ABOVE_GROUND_M) {
        terrain = h.terrain.loss_db(c.on_line);
        building = h.buildings.loss_db(c.on_segment);
    }
    double attenuation_gain = energy(screened_sel_db(0.0, lateral, terrain, building) - lateral);
    for (int p = 0; p < 3; ++p) {
        bool silent = true;
        for (int k = 0; k < ND; ++k) silent = silent && b.levels_db[p][k] == -INFINITY;
        if (silent) {
            out.sel_energy[p] = 0.0;
            continue;
        }
        double len = std::max(b.piece_length_m[p] * stretch, 1.0);
        double finite = finite_segment_energy_fraction(along + 0.5 * (len - c.length), len, scaled);
        out.sel_energy[p] = energy(box_level_db(b.levels_db[p], b.tail_levels_db[p], pos)) * finite * installation[p] *
                            attenuation_gain;
    }
    return out;
}

// boxes.rs:156-195
BoxSel box_sel_at_receiver(const BoxAtReceiver &a, const Horizons &h) {
    double length = average_length_m(*a.b);
    if (a.spread <= 0.0) return average_piece_sel(a, h, length);
    BoxAtReceiver lo = a, hi = a;
    lo.gradient = a.gradient - a.spread;
    hi.gradient = a.gradient + a.spread;
    BoxSel l = average_piece_sel(lo, h, length), u = average_piece_sel(hi, h, length), out;
    for (int p = 0; p < 3; ++p) {
        out.sel_energy[p] = 0.5 * (l.sel_energy[p] + u.sel_energy[p]);
        double le = l.sel_energy[p], ue = u.sel_energy[p];
        for (int k = 0; k < 3; ++k)
            out.fractions[p][k] = le + ue > 0.0 ? (le * l.fractions[p][k] + ue * u.fractions[p][k]) / (le + ue) : l.fractions[p][k];
    }
    return out;
}

// paint/src/flight_boxes.rs:24-33
double flight_weight(uint32_t kind, double distance_m, double coarse_m) {
    if (kind == QM_FLIGHT_WEIGHT_ONE) return 1.0;
    double f = std::min(std::max((distance_m - 1.5 * coarse_m) / (1.5 * coarse_m), 0.0), 1.0);
    double far = f * f * (3.0 - 2.0 * f);
    return kind == QM_FLIGHT_WEIGHT_FAR ? far : 1.0 - far;
}

// popup/src/aircraft.rs:86-95
void add_pass(double *class_energy, double *class_passing, int period, double e, double passing) {
    if (e <= 0.0 || passing <= 0.0) return;
    double level = 10.0 * std::log10(e / passing);
    // Rust's float-to-integer cast saturates: a level past the top class (an infinite one too) is the top class.
    double at = std::max((level - PASS_LOWEST_DB) / PASS_CLASS_DB, 0.0);
    int c = at >= (double)(PASS_CLASSES - 1) ? PASS_CLASSES - 1 : (int)at;
    class_energy[period * PASS_CLASSES + c] += e;
    class_passing[period * PASS_CLASSES + c] += passing;
}

// popup/src/aircraft/boxes.rs:187-223 box_at and :272-316 tile_flight_passes over one segment's boxes.
uint64_t segment_sums(const qm_flight_box *boxes, const qm_flight_point &pt, const float *horizons,
                      const qm_box_segment &s, double *sums) {
    Horizons h = Horizons::of(horizons);
    double reach = std::min(s.within_m, AIRCRAFT_REACH_M);
    double *class_energy = sums + 3, *class_passing = class_energy + 3 * PASS_CLASSES;
    uint64_t heard = 0;
    for (uint32_t k = 0; k < s.count; ++k) {
        const qm_flight_box &b = boxes[s.first + k];
        double east = b.east_m - pt.x, north = b.north_m - pt.y;
        double distance = std::hypot(east, north);
        double share = distance <= reach ? flight_weight(s.weight, distance, s.coarse_m) : 0.0;
        if (share <= 0.0) continue;
        ++heard;
        BoxAtReceiver a{{east, north, b.centroid_altitude_m - pt.altitude_m}, b.axis_rad, b.gradient, b.gradient_spread,
                        b.ground_m - pt.altitude_m, &b};
        BoxSel sel = box_sel_at_receiver(a, h);
        double impedance = b.helicopter ? 1.0 : pt.impedance_gain;
        for (int p = 0; p < 3; ++p) {
            double e = sel.sel_energy[p] * impedance / (PERIOD_HOURS_D[p] * 3600.0);
            sums[p] += share * e;
            add_pass(class_energy, class_passing, p, share * e, share * b.passing[p]);
        }
    }
    return heard;
}

template <class F>
void parallel_for(size_t n, int threads, F f) {
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < std::max(threads, 1); ++t)
        pool.emplace_back([&] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i);
            }
        });
    for (auto &th : pool) th.join();
}

}  // namespace

extern "C" {

double qmo_lateral_attenuation_db(double height_m, double lateral_m) { return lateral_attenuation_db(height_m, lateral_m); }
double qmo_speed_correction_db(double v_ref_kt, double speed_kt) { return speed_correction_db(v_ref_kt, speed_kt); }
double qmo_finite_segment_energy_fraction(double along_m, double length_m, double scaled_m) {
    return finite_segment_energy_fraction(along_m, length_m, scaled_m);
}
double qmo_installation_energy_gain(uint32_t installation, double height_m, double slant_m) {
    return installation_energy_gain(installation, height_m, slant_m);
}
double qmo_npd_level(const double *curve10, double slant_m, double tail_alpha) {
    return NpdPosition::at(slant_m).level(curve10, tail_alpha);
}
double qmo_tail_absorption(const double *sel10) { return tail_absorption_db_per_m(sel10); }

// The flight grid: per cell the total A-weighted SEL (lae), day-average third-octave levels
// (thirds[cells][28]) and Zwicker loudness (sone), over cells [cell_begin, cell_end).
void qmo_flight_grid(const qm_aircraft_type *types, uint32_t n_types, const qm_flight_segment *segs, size_t n_segs,
                     const qm_flight_grid_desc *g, uint32_t cell_begin, uint32_t cell_end, double *lae, double *thirds,
                     double *sone, int threads) {
    std::vector<Type> T(n_types);
    for (uint32_t t = 0; t < n_types; ++t) T[t] = make_type(types[t]);
    // Flight bounding boxes (horizontal) for the reach rule.
    uint32_t n_flights = 0;
    for (size_t i = 0; i < n_segs; ++i) n_flights = std::max(n_flights, segs[i].flight + 1);
    std::vector<double> box(4 * n_flights);
    for (uint32_t f = 0; f < n_flights; ++f) {
        box[4 * f] = box[4 * f + 1] = 1e300;
        box[4 * f + 2] = box[4 * f + 3] = -1e300;
    }
    for (size_t i = 0; i < n_segs; ++i) {
        const qm_flight_segment &s = segs[i];
        double *b = &box[4 * s.flight];
        b[0] = std::min({b[0], (double)s.start[0], (double)s.end[0]});
        b[1] = std::min({b[1], (double)s.start[1], (double)s.end[1]});
        b[2] = std::max({b[2], (double)s.start[0], (double)s.end[0]});
        b[3] = std::max({b[3], (double)s.start[1], (double)s.end[1]});
    }
    size_t cells = (size_t)g->nx * g->ny;
    if (cell_end <= cell_begin) {
        cell_begin = 0;
        cell_end = (uint32_t)cells;
    }
    parallel_for(cell_end - cell_begin, threads, [&](size_t k) {
        size_t cell = cell_begin + k;
        double rx = g->origin_m[0] + (double)(cell % g->nx) * g->spacing_m;
        double ry = g->origin_m[1] + (double)(cell / g->nx) * g->spacing_m;
        double rz = g->receiver_height_m;
        std::vector<double> e_type(n_types, 0.0);
        for (size_t i = 0; i < n_segs; ++i) {
            const qm_flight_segment &s = segs[i];
            if (g->reach_m > 0.0) {
                const double *b = &box[4 * s.flight];
                double dx = std::max({b[0] - rx, 0.0, rx - b[2]}), dy = std::max({b[1] - ry, 0.0, ry - b[3]});
                if (dx * dx + dy * dy > g->reach_m * g->reach_m) continue;
            }
            e_type[s.type] += energy(segment_sel_db(T[s.type], s, rx, ry, rz));
        }
        double total = 0.0;
        for (uint32_t t = 0; t < n_types; ++t) total += e_type[t];
        if (lae) lae[k] = total > 0.0 ? 10.0 * std::log10(total) : -INFINITY;
        double levels[28];
        for (int b = 0; b < 28; ++b) {
            double e = 0.0;
            for (uint32_t t = 0; t < n_types; ++t) e += e_type[t] * T[t].share[b];
            levels[b] = e > 0.0 ? 10.0 * std::log10(e / g->duration_s) : -INFINITY;
            if (thirds) thirds[k * 28 + b] = levels[b];
        }
        if (sone) sone[k] = qmo_zwicker(levels);
    });
}

// ---- Aircraft boxes ----------------------------------------------------------------------

double qmo_path_difference_loss_db(double delta) { return path_difference_loss_db(delta); }
double qmo_edge_loss_db(double er, double eh, double sr, double sh) { return edge_loss_db(er, eh, sr, sh); }
double qmo_screened_sel_db(double f, double l, double t, double b) { return screened_sel_db(f, l, t, b); }
double qmo_flight_weight(uint32_t kind, double distance_m, double coarse_m) { return flight_weight(kind, distance_m, coarse_m); }

// One horizon's loss toward p (east, north, up of the receiver) from its card floats.
double qmo_horizon_loss_db(const float *floats, int sectors, const double *p) {
    return SectorEdges{floats, sectors}.loss_db(p);
}

// The kernel's SEL of one segment at a receiver (the reference's segment_sel_at_receiver, no horizons).
double qmo_segment_sel_db(const qm_aircraft_type *type, const qm_flight_segment *g, double rx, double ry, double rz) {
    Type T = make_type(*type);
    return segment_sel_db(T, *g, rx, ry, rz);
}

// A box of `n` pieces (segments of `types`, each weighted per period by period_weights[3 n]) as
// the builder closes it (BoxSums::add, values). Returns 0 for a box without energy; position fields
// take the pieces' frame, ground_m, passing and helicopter stay as the caller set them.
int qmo_box_sums(const qm_aircraft_type *types, const qm_flight_segment *pieces, size_t n, const double *period_weights,
                 qm_flight_box *out) {
    BoxSums sums;
    for (size_t i = 0; i < n; ++i) {
        Type T = make_type(types[pieces[i].type]);
        double start[3] = {pieces[i].start[0], pieces[i].start[1], pieces[i].start[2]};
        double end[3] = {pieces[i].end[0], pieces[i].end[1], pieces[i].end[2]};
        sums.add(segment_energies(T, pieces[i]), T.installation, period_weights + 3 * i, start, end);
    }
    return sums.values(*out) ? 1 : 0;
}

// One box's SEL energies and installation fractions at a point (box_sel_at_receiver in the
// point's frame, as box_at places it); horizons nullable (free field).
void qmo_box_sel(const qm_flight_box *b, const qm_flight_point *pt, const float *horizons, double *sel_energy,
                 double *fractions) {
    BoxAtReceiver a{{b->east_m - pt->x, b->north_m - pt->y, b->centroid_altitude_m - pt->altitude_m},
                    b->axis_rad, b->gradient, b->gradient_spread, b->ground_m - pt->altitude_m, b};
    BoxSel sel = box_sel_at_receiver(a, Horizons::of(horizons));
    for (int p = 0; p < 3; ++p) {
        sel_energy[p] = sel.sel_energy[p];
        for (int k = 0; k < 3; ++k) fractions[3 * p + k] = sel.fractions[p][k];
    }
}

// Every request band's sums (FlightBoxes::sums per request: its segments in order, each box in
// order), sums[n_sums][QM_FLIGHT_SUMS] zeroed here; returns the boxes heard.
uint64_t qmo_flight_sums(const qm_flight_box *boxes, const qm_flight_point *points, const float *horizons,
                         const qm_box_segment *segments, size_t n_segments, double *sums, size_t n_sums, int threads) {
    std::vector<std::vector<uint32_t>> of_sum(n_sums);
    for (size_t i = 0; i < n_segments; ++i) of_sum[segments[i].sum].push_back((uint32_t)i);
    std::fill(sums, sums + n_sums * QM_FLIGHT_SUMS, 0.0);
    std::atomic<uint64_t> heard{0};
    parallel_for(n_sums, threads, [&](size_t k) {
        uint64_t mine = 0;
        for (uint32_t i : of_sum[k]) {
            const qm_box_segment &s = segments[i];
            const qm_flight_point &pt = points[s.point];
            mine += segment_sums(boxes, pt, horizons ? horizons + pt.horizons : nullptr, s, sums + k * QM_FLIGHT_SUMS);
        }
        heard += mine;
    });
    return heard.load();
}

}  // extern "C"
