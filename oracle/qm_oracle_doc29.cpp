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
    for (uint32_t t = 0; t < n_types; ++t) {
        T[t].v_ref_kt = types[t].v_ref_kt;
        T[t].installation = types[t].installation;
        for (int op = 0; op < 2; ++op)
            for (int r = 0; r < 10; ++r)
                T[t].rows[op][r] = make_row(types[t].sel_db[op][r], types[t].lamax_db[op][r], types[t].v_ref_kt);
        double weighted = 0.0;
        for (int b = 0; b < 28; ++b) weighted += energy(types[t].spectrum_db[b] + A_WEIGHTING_THIRDS[b]);
        for (int b = 0; b < 28; ++b) T[t].share[b] = energy(types[t].spectrum_db[b]) / weighted;
    }
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

}  // extern "C"
