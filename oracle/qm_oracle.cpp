// FP64 CPU oracle of the noise-map painter hot path — TEST INFRASTRUCTURE ONLY.
//
// A line-by-line restatement, in C++ and double precision, of the reference's CPU physics
// (the Rust crates `physics`, `popup`, `paint` of quietmap). Only the tests, the smoke check
// and the CPU-baseline leg of the benchmark load this library; the product path never does.
// Every function names the reference file:line it follows. Pinned against the reference's own
// known-answer tests (ISO/TR 17534-4 TC01-TC28 fixture, ray_tests.rs pins, atmosphere and
// Zwicker expectations) by tests/test_oracle.py.
//
// Input layout: the scene descriptor of include/qm_batch.h (lattice steps, x east, y north).

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <functional>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../include/qm_batch.h"

namespace {

constexpr int BANDS = 8;
constexpr int PERIODS = 3;
constexpr int SECTORS = 16;
constexpr double LN10 = 2.302585092994045684;
constexpr double PI = 3.141592653589793116;
constexpr double INF = std::numeric_limits<double>::infinity();

// physics/src/bands.rs:6-18
const double BAND_FREQUENCY_HZ[BANDS] = {63.0, 125.0, 250.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0};
constexpr double SPEED_OF_SOUND = 340.0;
const double PERIOD_HOURS[PERIODS] = {12.0, 4.0, 8.0};
const double PERIOD_PENALTY_DB[PERIODS] = {0.0, 5.0, 10.0};

// physics/src/bands.rs:34-41
inline double energy(double level_db) { return std::exp(level_db * (LN10 / 10.0)); }
inline double amplitude(double level_db) { return std::exp(level_db * (LN10 / 20.0)); }

// ---------------------------------------------------------------------------------------------
// Atmosphere: physics/src/atmosphere.rs:17-63
double exact_mid_band_frequency_hz(int band) { return 1000.0 * std::pow(10.0, 0.3 * (band - 4.0)); }

double alpha_db_per_km(double f, double temperature_c, double rh, double pressure_kpa) {
    const double temperature = temperature_c + 273.15;
    const double reference_temperature = 293.15, triple_point = 273.16;
    const double pressure_ratio = pressure_kpa / 101.325;
    const double saturation_exponent = -6.8346 * std::pow(triple_point / temperature, 1.261) + 4.6151;
    const double humidity = rh * std::pow(10.0, saturation_exponent) / pressure_ratio;
    const double oxygen = pressure_ratio * (24.0 + 4.04e4 * humidity * (0.02 + humidity) / (0.391 + humidity));
    const double t_ratio = temperature / reference_temperature;
    const double nitrogen = pressure_ratio * std::pow(t_ratio, -0.5) *
                            (9.0 + 280.0 * humidity * std::exp(-4.170 * (std::pow(t_ratio, -1.0 / 3.0) - 1.0)));
    const double f2 = f * f;
    return 8.686 * f2 *
           (1.84e-11 / pressure_ratio * std::sqrt(t_ratio) +
            std::pow(t_ratio, -2.5) * (0.01275 * std::exp(-2239.1 / temperature) / (oxygen + f2 / oxygen) +
                                       0.1068 * std::exp(-3352.0 / temperature) / (nitrogen + f2 / nitrogen))) *
           1000.0;
}

// ---------------------------------------------------------------------------------------------
// Vertical profile: physics/src/cnossos/mod.rs:22-83
struct VProfile {
    const double *d;
    const double *z;
    const double *g;
    size_t n;
};

// Rust `partition_point(|v| v <= x)`: first index with xs[i] > x.
inline size_t upper_le(const double *xs, size_t n, double x) { return std::upper_bound(xs, xs + n, x) - xs; }
// Rust `partition_point(|v| v < x)`: first index with xs[i] >= x.
inline size_t lower_lt(const double *xs, size_t n, double x) { return std::lower_bound(xs, xs + n, x) - xs; }

// physics/src/cnossos/mod.rs:63-83
double interpolate_with_steps(const double *xs, const double *ys, size_t n, double x, bool before) {
    if (x <= xs[0]) return ys[0];
    if (x >= xs[n - 1]) return ys[n - 1];
    size_t upper = before ? lower_lt(xs, n, x) : upper_le(xs, n, x);
    if (before && xs[upper] == x) return ys[upper];
    double x0 = xs[upper - 1], x1 = xs[upper];
    if (x1 == x0) return ys[upper];
    return ys[upper - 1] + (x - x0) / (x1 - x0) * (ys[upper] - ys[upper - 1]);
}

double ground_altitude_at(const VProfile &p, double x) { return interpolate_with_steps(p.d, p.z, p.n, x, false); }
double ground_altitude_before(const VProfile &p, double x) { return interpolate_with_steps(p.d, p.z, p.n, x, true); }

// physics/src/cnossos/mod.rs:42-58
double mean_ground_factor(const VProfile &p, double start_m, double end_m) {
    auto at = [&](double x, bool before) { return interpolate_with_steps(p.d, p.g, p.n, x, before); };
    if (end_m - start_m < 1e-3) return at(start_m, false);
    size_t first = upper_le(p.d, p.n, start_m);
    size_t last = lower_lt(p.d, p.n, end_m);
    double px = start_m, pg = at(start_m, false), total = 0.0;
    for (size_t i = first; i < last; ++i) {
        total += 0.5 * (pg + p.g[i]) * (p.d[i] - px);
        px = p.d[i];
        pg = p.g[i];
    }
    total += 0.5 * (pg + at(end_m, true)) * (end_m - px);
    return total / (end_m - start_m);
}

// ---------------------------------------------------------------------------------------------
// Mean planes: physics/src/cnossos/mean_plane.rs:19-120
struct MeanPlane {
    double slope, intercept;
    double altitude_at(double x) const { return slope * x + intercept; }
    double signed_height(double x, double z) const { return (z - altitude_at(x)) / std::sqrt(1.0 + slope * slope); }
    double projected_distance(double fx, double fz, double tx, double tz) const {
        return std::fabs((tx - fx) + slope * (tz - fz)) / std::sqrt(1.0 + slope * slope);
    }
    void mirror(double x, double z, double &ox, double &oz) const {
        double norm_sq = 1.0 + slope * slope;
        double offset = (z - altitude_at(x)) / norm_sq;
        ox = x + 2.0 * offset * slope;
        oz = z - 2.0 * offset;
    }
};

// physics/src/cnossos/mean_plane.rs:19-64
MeanPlane fit_mean_plane(const VProfile &p, double start_m, double end_m) {
    double reference_z = ground_altitude_at(p, start_m);
    double length = end_m - start_m;
    if (length < 1e-3) return MeanPlane{0.0, reference_z};
    double iz = 0.0, ixz = 0.0;
    auto accumulate = [&](double x0, double z0, double x1, double z1) {
        double u0 = x0 - start_m, u1 = x1 - start_m;
        double w0 = z0 - reference_z, w1 = z1 - reference_z;
        double width = u1 - u0;
        if (width <= 0.0) return;
        iz += 0.5 * (w0 + w1) * width;
        ixz += width * (u0 * (2.0 * w0 + w1) + u1 * (w0 + 2.0 * w1)) / 6.0;
    };
    size_t first = upper_le(p.d, p.n, start_m);
    size_t last = lower_lt(p.d, p.n, end_m);
    double px = start_m, pz = ground_altitude_at(p, start_m);
    for (size_t i = first; i < last; ++i) {
        accumulate(px, pz, p.d[i], p.z[i]);
        px = p.d[i];
        pz = p.z[i];
    }
    accumulate(px, pz, end_m, ground_altitude_before(p, end_m));
    double slope = 12.0 * (ixz - 0.5 * length * iz) / (length * length * length);
    double intercept_relative = iz / length - 0.5 * slope * length;
    return MeanPlane{slope, reference_z + intercept_relative - slope * start_m};
}

// physics/src/cnossos/mean_plane.rs:283-306
struct EqGeometry {
    MeanPlane plane;
    double zs, zr;
    bool source_below, receiver_below;
    double dp;
};

EqGeometry geometry_over(MeanPlane plane, double fx, double fz, double tx, double tz) {
    double hs = plane.signed_height(fx, fz), hr = plane.signed_height(tx, tz);
    return EqGeometry{plane, std::max(hs, 0.0), std::max(hr, 0.0), hs < 0.0, hr < 0.0,
                      plane.projected_distance(fx, fz, tx, tz)};
}

// ---------------------------------------------------------------------------------------------
// Ground attenuation: physics/src/cnossos/ground.rs:8-139
constexpr double SHORT_PATH_HEIGHT_FACTOR = 30.0;
constexpr double FAVOURABLE_CURVATURE_A0_PER_M = 2e-4;
constexpr double FAVOURABLE_TERRAIN_HEIGHT_COEFFICIENT = 6e-3;
constexpr double MINIMUM_HEIGHT_SUM_M = 1e-3;
constexpr double HARD_GROUND_BELOW = 1e-3;
enum State { HOMOGENEOUS = 0, FAVOURABLE = 1 };

struct GroundFactors {
    double path, impedance, floor;
};

// ground.rs:40-53
double ground_factor_near_source(const EqGeometry &g, double path_gf, double source_gf) {
    double height_sum = std::max(g.zs + g.zr, MINIMUM_HEIGHT_SUM_M);
    double ratio = g.dp / (SHORT_PATH_HEIGHT_FACTOR * height_sum);
    if (ratio <= 1.0) return path_gf * ratio + source_gf * (1.0 - ratio);
    return path_gf;
}

struct BandConstants {
    double f25, f15, f075, k;
};
const BandConstants *band_constants() {
    static BandConstants table[BANDS];
    static bool ready = [] {
        for (int b = 0; b < BANDS; ++b) {
            double f = BAND_FREQUENCY_HZ[b];
            table[b] = BandConstants{std::pow(f, 2.5), std::pow(f, 1.5), std::pow(f, 0.75),
                                     2.0 * PI * f / SPEED_OF_SOUND};
        }
        return true;
    }();
    (void)ready;
    return table;
}

// ground.rs:78-89
double analytic_ground_db(int band, double dp, double zs, double zr, double gw13) {
    const BandConstants &c = band_constants()[band];
    double k = c.k;
    double gw26 = gw13 * gw13;
    double w = 0.0185 * c.f25 * gw26 / (c.f15 * gw26 + 1.3e3 * c.f075 * gw13 + 1.16e6);
    double wd = w * dp;
    double cf = dp * (1.0 + 3.0 * wd * std::exp(-std::sqrt(wd))) / (1.0 + wd);
    double root = std::sqrt(2.0 * cf / k);
    double product = (zs * zs - root * zs + cf / k) * (zr * zr - root * zr + cf / k);
    return -10.0 * std::log10(4.0 * k * k / (dp * dp) * product);
}

// ground.rs:92-102
double favourable_floor_db(const EqGeometry &g, double floor_factor) {
    double height_sum = std::max(g.zs + g.zr, MINIMUM_HEIGHT_SUM_M);
    double base = -3.0 * (1.0 - floor_factor);
    double limit = SHORT_PATH_HEIGHT_FACTOR * height_sum;
    if (g.dp <= limit) return base;
    return base * (1.0 + 2.0 * (1.0 - limit / g.dp));
}

// ground.rs:105-139
void ground_attenuation_bands(const EqGeometry &g, GroundFactors f, int state, double out[BANDS]) {
    double dp = std::max(g.dp, 1e-6);
    double zs = g.zs, zr = g.zr;
    double gw13 = std::pow(std::max(f.impedance, 0.0), 1.3);
    if (state == HOMOGENEOUS) {
        if (f.path < HARD_GROUND_BELOW) {
            for (int b = 0; b < BANDS; ++b) out[b] = -3.0;
            return;
        }
        double floor = -3.0 * (1.0 - f.floor);
        for (int b = 0; b < BANDS; ++b) out[b] = std::max(analytic_ground_db(b, dp, zs, zr, gw13), floor);
    } else {
        double floor = favourable_floor_db(g, f.floor);
        if (f.path < HARD_GROUND_BELOW) {
            for (int b = 0; b < BANDS; ++b) out[b] = floor;
            return;
        }
        double height_sum = std::max(zs + zr, MINIMUM_HEIGHT_SUM_M);
        double curvature = FAVOURABLE_CURVATURE_A0_PER_M * dp * dp / 2.0;
        double terrain = FAVOURABLE_TERRAIN_HEIGHT_COEFFICIENT * dp / height_sum;
        double zsf = zs + curvature * (zs / height_sum) * (zs / height_sum) + terrain;
        double zrf = zr + curvature * (zr / height_sum) * (zr / height_sum) + terrain;
        for (int b = 0; b < BANDS; ++b) out[b] = std::max(analytic_ground_db(b, dp, zsf, zrf, gw13), floor);
    }
}

// ---------------------------------------------------------------------------------------------
// Rubber band: physics/src/cnossos/rubber_band.rs
struct PP {
    double x, z;
};
inline bool operator==(const PP &a, const PP &b) { return a.x == b.x && a.z == b.z; }

inline double distance(PP a, PP b) {
    double dx = b.x - a.x, dz = b.z - a.z;
    return std::sqrt(dx * dx + dz * dz);
}

// rubber_band.rs:352-364
double triangle_excess(PP s, PP o, PP r) {
    double ux = o.x - s.x, uz = o.z - s.z, vx = r.x - o.x, vz = r.z - o.z;
    double lu = std::sqrt(ux * ux + uz * uz), lv = std::sqrt(vx * vx + vz * vz);
    double wx = ux + vx, wz = uz + vz;
    double lw = std::sqrt(wx * wx + wz * wz);
    double dot = ux * vx + uz * vz;
    if (dot <= 0.0) return lu + lv - lw;
    double cross = ux * vz - uz * vx;
    return 2.0 * cross * cross / ((lu * lv + dot) * (lu + lv + lw));
}

// rubber_band.rs:366-369
inline double chord_altitude(PP from, PP to, double x) {
    return from.z + (to.z - from.z) * (x - from.x) / (to.x - from.x);
}

struct Sag {
    bool favourable;
    double along_per_x, chord, gamma2, centre_term;
    // rubber_band.rs:328-339
    double at(double x_from_source) const {
        if (!favourable) return 0.0;
        double along = x_from_source * along_per_x;
        double offset = along - 0.5 * chord;
        double perpendicular =
            along * (chord - along) / (std::sqrt(std::max(gamma2 - offset * offset, 0.0)) + centre_term);
        return perpendicular * along_per_x;
    }
};

// rubber_band.rs:207-317
struct StateRay {
    int state;
    double radius;

    static StateRay between(int state, PP s, PP r) {
        double direct = distance(s, r);
        return StateRay{state, std::max(1000.0, 8.0 * direct)};
    }
    double arc_excess(double chord) const {
        if (state == HOMOGENEOUS) return 0.0;
        double x = chord / (2.0 * radius);
        if (x > 1.0 / 16.0) return 2.0 * radius * std::asin(std::min(x, 1.0)) - chord;
        double x2 = x * x;
        return 2.0 * radius * x * x2 *
               (1.0 / 6.0 + x2 * (3.0 / 40.0 + x2 * (5.0 / 112.0 + x2 * (35.0 / 1152.0))));
    }
    double length(PP a, PP b) const {
        double chord = distance(a, b);
        return chord + arc_excess(chord);
    }
    double path_difference(PP from, const PP *points, size_t n, PP to) const {
        if (n == 0) return 0.0;
        PP first = points[0];
        double chords = 0.0, arcs = 0.0;
        PP start = from;
        for (size_t i = 0; i < n; ++i) {
            chords += triangle_excess(start, points[i], to);
            arcs += arc_excess(distance(start, points[i]));
            start = points[i];
        }
        arcs += arc_excess(distance(start, to)) - arc_excess(distance(from, to));
        double excess = chords + arcs;
        if (n > 1) return excess;
        double chord = chord_altitude(from, to, first.x);
        if (state == HOMOGENEOUS) return first.z >= chord ? excess : -excess;
        if (first.z >= chord) return excess;
        PP on_chord{first.x, chord};
        return 2.0 * triangle_excess(from, on_chord, to) - triangle_excess(from, first, to) +
               2.0 * arc_excess(distance(from, on_chord)) + 2.0 * arc_excess(distance(on_chord, to)) -
               arc_excess(distance(from, first)) - arc_excess(distance(first, to)) -
               arc_excess(distance(from, to));
    }
    Sag sag(PP source, PP receiver) const {
        double horizontal = receiver.x - source.x;
        double chord = distance(source, receiver);
        double gamma2 = radius * radius;
        return Sag{state == FAVOURABLE, chord / horizontal, chord, gamma2,
                   std::sqrt(gamma2 - 0.25 * chord * chord)};
    }
};

struct Blocking {
    double x, z;
    size_t index;
};

// rubber_band.rs:373-444
void diffraction_path(const StateRay &ray, PP source, PP receiver, const std::vector<PP> &candidates,
                      std::vector<Blocking> &blocking, std::vector<Blocking> &hull, std::vector<PP> &points,
                      bool &blocked) {
    points.clear();
    blocked = false;
    blocking.clear();
    Sag sag = ray.sag(source, receiver);
    for (size_t index = 0; index < candidates.size(); ++index) {
        double x = candidates[index].x, z = candidates[index].z;
        if (z > chord_altitude(source, receiver, x) + sag.at(x - source.x)) {
            if (!blocking.empty() && blocking.back().x == x) {
                if (z > blocking.back().z) blocking.back() = Blocking{x, z, index};
            } else {
                blocking.push_back(Blocking{x, z, index});
            }
        }
    }
    if (!blocking.empty()) {
        blocked = true;
        hull.clear();
        const size_t none = SIZE_MAX;
        auto push = [&](Blocking point) {
            while (hull.size() >= 2) {
                Blocking a = hull[hull.size() - 2], b = hull[hull.size() - 1];
                PP from{a.x, a.z}, to{point.x, point.z};
                double ray_at_b = chord_altitude(from, to, b.x) + ray.sag(from, to).at(b.x - a.x);
                if (b.z <= ray_at_b)
                    hull.pop_back();
                else
                    break;
            }
            hull.push_back(point);
        };
        push(Blocking{source.x, source.z, none});
        for (const Blocking &b : blocking) push(b);
        push(Blocking{receiver.x, receiver.z, none});
        for (size_t i = 1; i + 1 < hull.size(); ++i) points.push_back(candidates[hull[i].index]);
        return;
    }
    bool have = false;
    double best_value = 0.0;
    PP best{};
    for (const PP &c : candidates) {
        double delta = ray.path_difference(source, &c, 1, receiver);
        if (!have || delta > best_value) {
            have = true;
            best_value = delta;
            best = c;
        }
    }
    if (have) points.push_back(best);
}

// ---------------------------------------------------------------------------------------------
// Diffraction: physics/src/cnossos/diffraction.rs
constexpr double DIFFRACTION_CAP_DB = 25.0;
constexpr double MULTIPLE_DIFFRACTION_MINIMUM_SPAN_M = 0.3;

// diffraction.rs:19-29
void diffraction_db(double delta, const double c2[BANDS], double out[BANDS]) {
    for (int b = 0; b < BANDS; ++b) {
        double lambda = SPEED_OF_SOUND / BAND_FREQUENCY_HZ[b];
        double x = 40.0 * c2[b] * delta / lambda;
        out[b] = x >= -2.0 ? 10.0 * std::log10(3.0 + x) : 0.0;
    }
}

// diffraction.rs:32-34
double ground_split_db(double ground_db, double mirrored_db, double direct_db) {
    return -20.0 * std::log10(1.0 + (amplitude(-ground_db) - 1.0) * amplitude(-(mirrored_db - direct_db)));
}

struct VPath {
    VProfile profile;
    PP source, receiver;
    double source_ground_factor;
    const PP *terrain;
    size_t n_terrain;
    const PP *tops;
    size_t n_tops;
};

struct DirectPath {
    EqGeometry geometry;
    double path_ground, near_source;
};

// diffraction.rs:44-61
DirectPath direct_path_of(const VPath &path) {
    double length = path.receiver.x;
    EqGeometry g = geometry_over(fit_mean_plane(path.profile, 0.0, length), path.source.x, path.source.z,
                                 path.receiver.x, path.receiver.z);
    double pg = mean_ground_factor(path.profile, 0.0, length);
    return DirectPath{g, pg, ground_factor_near_source(g, pg, path.source_ground_factor)};
}

// diffraction.rs:200-213
GroundFactors source_side_factors(int state, double path_ground, double near_source) {
    return GroundFactors{path_ground, state == HOMOGENEOUS ? near_source : path_ground, near_source};
}

struct StateBoundary {
    double attenuation[BANDS];
    double without_ground[BANDS];
};

struct PathScratch {
    std::vector<PP> candidates;
    std::vector<Blocking> blocking, hull;
    std::vector<PP> points;
};

// diffraction.rs:64-197
StateBoundary boundary_for_candidates(const VPath &path, int state, const DirectPath &shared, PathScratch &s) {
    PP source = path.source, receiver = path.receiver;
    double length = receiver.x;
    const VProfile &profile = path.profile;
    StateBoundary boundary;
    ground_attenuation_bands(shared.geometry, source_side_factors(state, shared.path_ground, shared.near_source),
                             state, boundary.attenuation);
    for (int b = 0; b < BANDS; ++b) boundary.without_ground[b] = 0.0;
    StateRay ray = StateRay::between(state, source, receiver);
    bool blocked = false;
    diffraction_path(ray, source, receiver, s.candidates, s.blocking, s.hull, s.points, blocked);
    const std::vector<PP> &points = s.points;
    if (points.empty()) return boundary;
    PP first = points.front(), last = points.back();
    double delta = ray.path_difference(source, points.data(), points.size(), receiver);
    double span = 0.0;
    if (points.size() > 1)
        for (size_t i = 0; i + 1 < points.size(); ++i) span += ray.length(points[i], points[i + 1]);
    double c2[BANDS];
    for (int b = 0; b < BANDS; ++b) {
        if (points.size() > 1 && span > MULTIPLE_DIFFRACTION_MINIMUM_SPAN_M) {
            double x = 5.0 * SPEED_OF_SOUND / BAND_FREQUENCY_HZ[b] / span;
            c2[b] = (1.0 + x * x) / (1.0 / 3.0 + x * x);
        } else {
            c2[b] = 1.0;
        }
    }
    EqGeometry source_side = geometry_over(fit_mean_plane(profile, 0.0, first.x), source.x, source.z, first.x, first.z);
    EqGeometry receiver_side =
        geometry_over(fit_mean_plane(profile, last.x, length), last.x, last.z, receiver.x, receiver.z);
    PP source_image, receiver_image;
    source_side.plane.mirror(source.x, source.z, source_image.x, source_image.z);
    receiver_side.plane.mirror(receiver.x, receiver.z, receiver_image.x, receiver_image.z);
    double direct_db[BANDS], source_image_db[BANDS], receiver_image_db[BANDS];
    diffraction_db(delta, c2, direct_db);
    diffraction_db(ray.path_difference(source_image, points.data(), points.size(), receiver), c2, source_image_db);
    diffraction_db(ray.path_difference(source, points.data(), points.size(), receiver_image), c2, receiver_image_db);
    double source_side_ground = mean_ground_factor(profile, 0.0, first.x);
    double source_side_near = ground_factor_near_source(source_side, source_side_ground, path.source_ground_factor);
    double ground_so[BANDS], ground_or[BANDS];
    ground_attenuation_bands(source_side, source_side_factors(state, source_side_ground, source_side_near), state,
                             ground_so);
    double receiver_side_ground = mean_ground_factor(profile, last.x, length);
    ground_attenuation_bands(receiver_side,
                             GroundFactors{receiver_side_ground, receiver_side_ground, receiver_side_ground}, state,
                             ground_or);
    double rayleigh_star =
        blocked ? 0.0 : ray.path_difference(source_image, points.data(), points.size(), receiver_image);
    for (int b = 0; b < BANDS; ++b) {
        double lambda = SPEED_OF_SOUND / BAND_FREQUENCY_HZ[b];
        bool admitted = blocked || (delta > -lambda / 20.0 && delta > lambda / 4.0 - rayleigh_star);
        if (!admitted) continue;
        double sr = direct_db[b];
        double ground_free = std::min(std::max(sr, 0.0), DIFFRACTION_CAP_DB);
        double split_so;
        if (source_side.source_below) {
            sr = source_image_db[b];
            split_so = ground_so[b];
        } else {
            split_so = ground_split_db(ground_so[b], source_image_db[b], direct_db[b]);
        }
        if (!std::isfinite(split_so)) {
            split_so = ground_so[b];
            sr = source_image_db[b];
        }
        double split_or;
        if (receiver_side.receiver_below) {
            sr = receiver_image_db[b];
            split_or = ground_or[b];
        } else {
            split_or = ground_split_db(ground_or[b], receiver_image_db[b], sr);
        }
        if (!std::isfinite(split_or)) {
            split_or = ground_or[b];
            sr = receiver_image_db[b];
        }
        boundary.attenuation[b] = std::min(std::max(sr, 0.0), DIFFRACTION_CAP_DB) + split_so + split_or;
        boundary.without_ground[b] = ground_free;
    }
    return boundary;
}

// physics/src/cnossos/mod.rs:154-176
void collect_candidates(const VPath &path, std::vector<PP> &out) {
    out.clear();
    double length = path.receiver.x;
    auto inside = [&](const PP &p) { return p.x > 0.0 && p.x < length; };
    size_t i = 0, j = 0;
    auto skip_t = [&] {
        while (i < path.n_terrain && !inside(path.terrain[i])) ++i;
    };
    auto skip_o = [&] {
        while (j < path.n_tops && !inside(path.tops[j])) ++j;
    };
    skip_t();
    skip_o();
    while (i < path.n_terrain || j < path.n_tops) {
        if (i < path.n_terrain && j < path.n_tops) {
            if (path.tops[j].x < path.terrain[i].x) {
                out.push_back(path.tops[j++]);
            } else {
                out.push_back(path.terrain[i++]);
            }
        } else if (i < path.n_terrain) {
            out.push_back(path.terrain[i++]);
        } else {
            out.push_back(path.tops[j++]);
        }
        skip_t();
        skip_o();
    }
}

// physics/src/cnossos/mod.rs:123-133
void state_boundaries(const VPath &path, PathScratch &s, StateBoundary out[2], bool want_favourable = true) {
    collect_candidates(path, s.candidates);
    DirectPath direct = direct_path_of(path);
    out[0] = boundary_for_candidates(path, HOMOGENEOUS, direct, s);
    if (want_favourable) {
        out[1] = boundary_for_candidates(path, FAVOURABLE, direct, s);
    } else {
        out[1] = out[0];
    }
}

// ---------------------------------------------------------------------------------------------
// One ray: physics/src/ray.rs
constexpr double CREST_ENDS_M = 300.0;
constexpr double CREST_SPACING_M = 150.0;

struct Crossing {
    double t;
    double height_m;
    bool building;
    bool bounds_roof;
    uint64_t footprint_id;
    uint32_t edge;  // first vertex of the crossed edge (for listing; not part of the physics)
};

struct Profile {
    double horizontal_m;
    std::vector<double> t, ground_m, ground_factor;
    void clear(double horizontal) {
        horizontal_m = horizontal;
        t.clear();
        ground_m.clear();
        ground_factor.clear();
    }
    void push(double tt, double z, double g) {
        t.push_back(tt);
        ground_m.push_back(z);
        ground_factor.push_back(g);
    }
};

struct RayEnds {
    double source_height_m;
    bool has_source_ground;
    double source_ground_m;
    double receiver_altitude_m;
    bool has_source_ground_factor;
    double source_ground_factor;
    double platform_half_width_m;
    uint64_t own_footprint;
};

struct Transfer {
    double slant_m;
    double periods[PERIODS][BANDS];
    double states[2][BANDS];
};

struct Roof {
    double x0, x1, top0, top1;
};

struct Building {
    uint64_t id;
    double x, top;
};

struct PathBuffers {
    std::vector<double> d, z, g;
    std::vector<PP> terrain, crests, tops;
    std::vector<Roof> roofs;
    std::vector<Building> buildings;
    std::vector<uint64_t> containing;
};

// ray.rs:406-417
double interpolate_pp(const std::vector<PP> &points, double at) {
    size_t n = points.size();
    size_t upper = std::upper_bound(points.begin(), points.end(), at,
                                    [](double v, const PP &p) { return v < p.x; }) -
                   points.begin();
    upper = std::min(std::max(upper, (size_t)1), n - 1);
    PP a = points[upper - 1], b = points[upper];
    double f = b.x > a.x ? std::min(std::max((at - a.x) / (b.x - a.x), 0.0), 1.0) : 0.0;
    return a.z + f * (b.z - a.z);
}

// ray.rs:201-226
void containing_footprints(const std::vector<Crossing> &crossings, uint64_t own, std::vector<uint64_t> &out) {
    out.clear();
    if (own == 0) return;
    for (const Crossing &c : crossings)
        if (c.bounds_roof) out.push_back(c.footprint_id);
    std::sort(out.begin(), out.end());
    size_t odd = 0, start = 0;
    while (start < out.size()) {
        uint64_t id = out[start];
        size_t end = start;
        while (end < out.size() && out[end] == id) ++end;
        if ((end - start) % 2 == 1) out[odd++] = id;
        start = end;
    }
    out.resize(odd);
    out.push_back(own);
    std::sort(out.begin(), out.end());
}

// ray.rs:360-385
void crests_of(const std::vector<PP> &terrain, double length, std::vector<PP> &out) {
    out.clear();
    auto middle = [&](double x) { return x > CREST_ENDS_M && x < length - CREST_ENDS_M; };
    bool open = false;
    PP best{};
    int64_t at = 0;
    for (const PP &point : terrain) {
        int64_t group = (int64_t)std::floor(point.x / CREST_SPACING_M);
        if (open && (!middle(point.x) || at != group)) {
            out.push_back(best);
            open = false;
        }
        if (!middle(point.x)) {
            out.push_back(point);
            continue;
        }
        if (open && point.z <= best.z) {
            // keep
        } else {
            open = true;
            best = point;
            at = group;
        }
    }
    if (open) out.push_back(best);
}

// ray.rs:389-404
void clip_roofs_in_closing_order(std::vector<Roof> &roofs) {
    std::stable_sort(roofs.begin(), roofs.end(), [](const Roof &a, const Roof &b) {
        if (a.x1 != b.x1) return a.x1 < b.x1;
        return a.x0 < b.x0;
    });
    double covered_to = -INF;
    size_t kept = 0;
    for (size_t i = 0; i < roofs.size(); ++i) {
        Roof roof = roofs[i];
        if (roof.x1 <= covered_to) continue;
        if (roof.x0 < covered_to) {
            double span = roof.x1 - roof.x0;
            roof.top0 += (covered_to - roof.x0) / span * (roof.top1 - roof.top0);
            roof.x0 = covered_to;
        }
        covered_to = roof.x1;
        roofs[kept++] = roof;
    }
    roofs.resize(kept);
}

// ray.rs:255-354
void fill_path(PathBuffers &pb, const Profile &profile, const std::vector<Crossing> &crossings, const RayEnds &ends) {
    double length = std::max(profile.horizontal_m, 1.0);
    pb.terrain.clear();
    double source_ground = ends.has_source_ground ? ends.source_ground_m : profile.ground_m[0];
    for (size_t i = 0; i < profile.t.size(); ++i) {
        double x = profile.t[i] * length;
        double z = profile.ground_m[i];
        pb.terrain.push_back(PP{x, x < ends.platform_half_width_m ? std::min(z, source_ground) : z});
    }
    crests_of(pb.terrain, length, pb.crests);
    const std::vector<PP> &terrain = pb.terrain;
    auto terrain_at = [&](double x) { return interpolate_pp(terrain, x); };
    auto ground_factor_at = [&](double x) {
        size_t n = terrain.size();
        size_t upper = std::upper_bound(terrain.begin(), terrain.end(), x,
                                        [](double v, const PP &p) { return v < p.x; }) -
                       terrain.begin();
        upper = std::min(std::max(upper, (size_t)1), n - 1);
        double x0 = terrain[upper - 1].x, x1 = terrain[upper].x;
        double f = x1 > x0 ? std::min(std::max((x - x0) / (x1 - x0), 0.0), 1.0) : 0.0;
        double a = profile.ground_factor[upper - 1], b = profile.ground_factor[upper];
        return a + f * (b - a);
    };
    pb.tops.clear();
    pb.roofs.clear();
    pb.buildings.clear();
    containing_footprints(crossings, ends.own_footprint, pb.containing);
    for (const Crossing &c : crossings) {
        if (std::binary_search(pb.containing.begin(), pb.containing.end(), c.footprint_id)) continue;
        double x = c.t * length;
        double top = terrain_at(x) + c.height_m;
        pb.tops.push_back(PP{x, top});
        if (c.bounds_roof) pb.buildings.push_back(Building{c.footprint_id, x, top});
    }
    std::stable_sort(pb.buildings.begin(), pb.buildings.end(), [](const Building &a, const Building &b) {
        if (a.id != b.id) return a.id < b.id;
        return a.x < b.x;
    });
    for (size_t start = 0; start < pb.buildings.size();) {
        size_t end = start;
        while (end < pb.buildings.size() && pb.buildings[end].id == pb.buildings[start].id) ++end;
        for (size_t k = start; k + 1 < end; k += 2)
            pb.roofs.push_back(Roof{pb.buildings[k].x, pb.buildings[k + 1].x, pb.buildings[k].top,
                                    pb.buildings[k + 1].top});
        start = end;
    }
    clip_roofs_in_closing_order(pb.roofs);
    pb.d.clear();
    pb.z.clear();
    pb.g.clear();
    auto push = [&](double x, double altitude, double ground) {
        pb.d.push_back(x);
        pb.z.push_back(altitude);
        pb.g.push_back(ground);
    };
    push(0.0, terrain[0].z, profile.ground_factor[0]);
    size_t r = 0;
    double covered_to = 0.0;
    for (size_t index = 1; index < terrain.size(); ++index) {
        double x = terrain[index].x, altitude = terrain[index].z;
        while (r < pb.roofs.size()) {
            const Roof &roof = pb.roofs[r];
            if (roof.x0 >= x) break;
            push(roof.x0, terrain_at(roof.x0), ground_factor_at(roof.x0));
            push(roof.x0, roof.top0, 0.0);
            push(roof.x1, roof.top1, 0.0);
            push(roof.x1, terrain_at(roof.x1), ground_factor_at(roof.x1));
            covered_to = roof.x1;
            ++r;
        }
        if (x > covered_to) push(x, altitude, profile.ground_factor[index]);
    }
}

struct RayScratch {
    PathBuffers pb;
    PathScratch ps;
};

inline double attenuation_energy(double db) { return std::exp(-db * (LN10 / 10.0)); }

// ray.rs:125-191 (foliage is zero: the synthetic scenes carry no tree cover)
void ray_terms(const Profile &profile, const std::vector<Crossing> &crossings, const RayEnds &ends,
               const double p[PERIODS], const double alpha[BANDS], RayScratch &scratch, Transfer &out,
               StateBoundary boundaries[2], bool want_favourable = true) {
    double horizontal = std::max(profile.horizontal_m, 1.0);
    double source_altitude =
        (ends.has_source_ground ? ends.source_ground_m : profile.ground_m[0]) + ends.source_height_m;
    double slant = std::max(std::hypot(horizontal, ends.receiver_altitude_m - source_altitude), 1.0);
    fill_path(scratch.pb, profile, crossings, ends);
    const PathBuffers &pb = scratch.pb;
    double length = pb.d.back();
    VPath path;
    path.profile = VProfile{pb.d.data(), pb.z.data(), pb.g.data(), pb.d.size()};
    path.source = PP{0.0, source_altitude};
    path.receiver = PP{length, ends.receiver_altitude_m};
    path.source_ground_factor = ends.has_source_ground_factor ? ends.source_ground_factor : profile.ground_factor[0];
    path.terrain = pb.crests.data();
    path.n_terrain = pb.crests.size();
    path.tops = pb.tops.data();
    path.n_tops = pb.tops.size();
    state_boundaries(path, scratch.ps, boundaries, want_favourable);
    double air[BANDS];
    for (int b = 0; b < BANDS; ++b) air[b] = attenuation_energy(alpha[b] * slant / 1000.0);
    double hom[BANDS], fav[BANDS];
    for (int b = 0; b < BANDS; ++b) {
        hom[b] = attenuation_energy(boundaries[0].attenuation[b]);
        fav[b] = attenuation_energy(boundaries[1].attenuation[b]);
    }
    out.slant_m = slant;
    for (int period = 0; period < PERIODS; ++period)
        for (int b = 0; b < BANDS; ++b)
            out.periods[period][b] = air[b] * (p[period] * fav[b] + (1.0 - p[period]) * hom[b]);
    for (int b = 0; b < BANDS; ++b) {
        out.states[0][b] = air[b] * hom[b];
        out.states[1][b] = air[b] * fav[b];
    }
}

// ---------------------------------------------------------------------------------------------
// Weather: physics/src/weather.rs:61-70
double favourable_at(const float row[SECTORS], double azimuth_rad) {
    double bearing = std::fmod(90.0 - azimuth_rad * (180.0 / PI), 360.0);
    if (bearing < 0.0) bearing += 360.0;  // rem_euclid
    if (bearing >= 360.0) bearing -= 360.0;
    double position = bearing / (360.0 / SECTORS);
    size_t lower = (size_t)std::floor(position) % SECTORS;
    size_t upper = (lower + 1) % SECTORS;
    double fraction = position - std::floor(position);
    return row[lower] + fraction * (row[upper] - row[lower]);
}

// ---------------------------------------------------------------------------------------------
// Scene: obstacles with a uniform cell grid, terrain, sources.
struct Scene {
    double step_m;
    int64_t cell_steps;
    int64_t cells_x, cells_y;
    std::vector<int32_t> vertices;  // [n][2]
    std::vector<qm_outline> outlines;
    std::vector<uint32_t> cell_start;  // CSR over cells_y*cells_x
    std::vector<uint32_t> cell_edges;  // (outline << 0) packed as pairs: edge start vertex, outline index
    std::vector<uint32_t> cell_outline;
    // terrain
    int dem_nx, dem_ny;
    int64_t dem_ox, dem_oy, dem_spacing;
    std::vector<float> dem_z, dem_g;
    double flat_z, flat_g;
    std::vector<qm_source> sources;
    float favourable[PERIODS][SECTORS];
    double alpha[BANDS];
};

// Whether the closed segment a-b meets the closed box [x0, x1] x [y0, y1] (exact integers).
bool segment_meets_box(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t x0, int64_t y0, int64_t x1,
                       int64_t y1) {
    if (std::max(ax, bx) < x0 || std::min(ax, bx) > x1 || std::max(ay, by) < y0 || std::min(ay, by) > y1)
        return false;
    int64_t dx = bx - ax, dy = by - ay;
    auto side = [&](int64_t px, int64_t py) {
        int64_t c = dx * (py - ay) - dy * (px - ax);
        return (c > 0) - (c < 0);
    };
    int s0 = side(x0, y0), s1 = side(x1, y0), s2 = side(x0, y1), s3 = side(x1, y1);
    if (s0 > 0 && s1 > 0 && s2 > 0 && s3 > 0) return false;
    if (s0 < 0 && s1 < 0 && s2 < 0 && s3 < 0) return false;
    return true;
}

// The cell lists: every edge in every cell whose closed box it meets (a supercover), so every
// point of an edge lies in a cell that lists it (the builder's rule, tiles::obstacles).
void build_cells(Scene &s) {
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> lists(s.cells_x * s.cells_y);
    int64_t C = s.cell_steps;
    for (uint32_t o = 0; o < s.outlines.size(); ++o) {
        const qm_outline &ol = s.outlines[o];
        for (uint32_t k = 0; k + 1 < ol.vertex_count; ++k) {
            uint32_t e = ol.first_vertex + k;
            int64_t ax = s.vertices[2 * e], ay = s.vertices[2 * e + 1];
            int64_t bx = s.vertices[2 * e + 2], by = s.vertices[2 * e + 3];
            int64_t cx0 = std::max<int64_t>(0, (int64_t)std::floor((double)std::min(ax, bx) / C) - 1);
            int64_t cx1 = std::min<int64_t>(s.cells_x - 1, (int64_t)std::floor((double)std::max(ax, bx) / C) + 1);
            int64_t cy0 = std::max<int64_t>(0, (int64_t)std::floor((double)std::min(ay, by) / C) - 1);
            int64_t cy1 = std::min<int64_t>(s.cells_y - 1, (int64_t)std::floor((double)std::max(ay, by) / C) + 1);
            for (int64_t cy = cy0; cy <= cy1; ++cy)
                for (int64_t cx = cx0; cx <= cx1; ++cx)
                    if (segment_meets_box(ax, ay, bx, by, cx * C, cy * C, (cx + 1) * C, (cy + 1) * C))
                        lists[cy * s.cells_x + cx].push_back({e, o});
        }
    }
    s.cell_start.assign(lists.size() + 1, 0);
    s.cell_edges.clear();
    s.cell_outline.clear();
    for (size_t c = 0; c < lists.size(); ++c) {
        s.cell_start[c] = (uint32_t)s.cell_edges.size();
        for (auto &pr : lists[c]) {
            s.cell_edges.push_back(pr.first);
            s.cell_outline.push_back(pr.second);
        }
    }
    s.cell_start[lists.size()] = (uint32_t)s.cell_edges.size();
}

// popup/src/obstacles/crossings.rs:13-28
bool segment_intersection_t(const double start[2], const double delta[2], const double a[2], const double b[2],
                            double &t_out) {
    double ex = b[0] - a[0], ey = b[1] - a[1];
    double denominator = delta[0] * ey - delta[1] * ex;
    if (denominator == 0.0) return false;
    double wx = a[0] - start[0], wy = a[1] - start[1];
    double t = (wx * ey - wy * ex) / denominator;
    double u = (wx * delta[1] - wy * delta[0]) / denominator;
    if (t > 0.0 && t < 1.0 && u >= 0.0 && u <= 1.0) {
        t_out = t;
        return true;
    }
    return false;
}

// popup/src/obstacles/crossings.rs:34-56 (sort_unstable_by (t, footprint); equal keys are merged)
void sort_and_deduplicate(std::vector<Crossing> &c) {
    std::sort(c.begin(), c.end(), [](const Crossing &a, const Crossing &b) {
        if (a.t != b.t) return a.t < b.t;
        if (a.footprint_id != b.footprint_id) return a.footprint_id < b.footprint_id;
        return a.edge < b.edge;
    });
    size_t kept = 0;
    for (size_t i = 0; i < c.size(); ++i) {
        Crossing candidate = c[i];
        bool merged = false;
        for (size_t k = kept; k-- > 0;) {
            if (!(candidate.t - c[k].t < 1e-9)) break;
            if (c[k].footprint_id == candidate.footprint_id) {
                c[k].bounds_roof = c[k].bounds_roof || candidate.bounds_roof;
                merged = true;
                break;
            }
        }
        if (!merged) c[kept++] = candidate;
    }
    c.resize(kept);
}

// popup/src/obstacles/crossings.rs:80-111
bool edge_bounds_roof(const Scene &s, const double start[2], const double delta[2], size_t edge, size_t first,
                      size_t count) {
    auto side = [&](size_t index) {
        double vx = s.vertices[2 * index], vy = s.vertices[2 * index + 1];
        return delta[0] * (vy - start[1]) - delta[1] * (vx - start[0]);
    };
    double a = side(edge), b = side(edge + 1);
    if (a != 0.0 && b != 0.0) return true;
    size_t distinct = count - 1;
    size_t vertex = ((a == 0.0 ? edge : edge + 1) - first) % distinct;
    double neighbours[2] = {0.0, 0.0};
    for (size_t offset = 1; offset < distinct; ++offset) {
        if (neighbours[0] == 0.0) neighbours[0] = side(first + (vertex + distinct - offset) % distinct);
        if (neighbours[1] == 0.0) neighbours[1] = side(first + (vertex + offset) % distinct);
        if (neighbours[0] != 0.0 && neighbours[1] != 0.0) break;
    }
    return neighbours[0] * neighbours[1] < 0.0;
}

// popup/src/obstacles/crossings.rs:163-226, over the scene's one uniform grid.
void scene_crossings(const Scene &s, const double from[2], const double to[2], std::vector<Crossing> &out,
                     uint64_t *edges_tested = nullptr) {
    out.clear();
    double start[2] = {from[0], from[1]};
    double end[2] = {to[0], to[1]};
    double delta[2] = {end[0] - start[0], end[1] - start[1]};
    double cell_steps = (double)s.cell_steps;
    int64_t cell[2] = {(int64_t)std::floor(start[0] / cell_steps), (int64_t)std::floor(start[1] / cell_steps)};
    int64_t last[2] = {(int64_t)std::floor(end[0] / cell_steps), (int64_t)std::floor(end[1] / cell_steps)};
    int64_t step[2] = {delta[0] >= 0.0 ? 1 : -1, delta[1] >= 0.0 ? 1 : -1};
    double t_delta[2], t_max[2];
    for (int axis = 0; axis < 2; ++axis) {
        t_delta[axis] = delta[axis] != 0.0 ? std::fabs(cell_steps / delta[axis]) : INF;
        if (delta[axis] == 0.0) {
            t_max[axis] = INF;
        } else {
            double boundary = (double)(cell[axis] + (delta[axis] >= 0.0 ? 1 : 0)) * cell_steps;
            t_max[axis] = std::fabs((boundary - start[axis]) / delta[axis]);
        }
    }
    double pad = 1e-9 * (1.0 + std::fabs(delta[0]) + std::fabs(delta[1]));
    auto along = [&](double t, double p[2]) {
        p[0] = start[0] + delta[0] * t;
        p[1] = start[1] + delta[1] * t;
    };
    double t_enter = 0.0;
    for (;;) {
        if (cell[0] >= 0 && cell[1] >= 0 && cell[0] < s.cells_x && cell[1] < s.cells_y) {
            size_t c = (size_t)(cell[1] * s.cells_x + cell[0]);
            uint32_t b = s.cell_start[c], e = s.cell_start[c + 1];
            if (b < e) {
                double t_exit = std::min(std::min(t_max[0], t_max[1]), 1.0);
                double p[2], q[2];
                along(std::min(std::max(t_enter, 0.0), 1.0), p);
                along(std::min(std::max(t_exit, 0.0), 1.0), q);
                // piece_box, crossings.rs:60-67
                int64_t low[2], high[2];
                for (int axis = 0; axis < 2; ++axis) {
                    low[axis] = (int64_t)std::floor(std::min(p[axis], q[axis]) - pad);
                    high[axis] = (int64_t)std::ceil(std::max(p[axis], q[axis]) + pad);
                }
                for (uint32_t k = b; k < e; ++k) {
                    uint32_t edge = s.cell_edges[k], o = s.cell_outline[k];
                    int64_t ax = s.vertices[2 * edge], ay = s.vertices[2 * edge + 1];
                    int64_t bx = s.vertices[2 * edge + 2], by = s.vertices[2 * edge + 3];
                    // edge_meets_box, crossings.rs:70-75
                    bool meets = high[0] >= std::min(ax, bx) && std::max(ax, bx) >= low[0] &&
                                 high[1] >= std::min(ay, by) && std::max(ay, by) >= low[1];
                    if (!meets) continue;
                    if (edges_tested) ++*edges_tested;
                    double a[2] = {(double)ax, (double)ay}, bb[2] = {(double)bx, (double)by};
                    double t;
                    if (segment_intersection_t(start, delta, a, bb, t)) {
                        const qm_outline &record = s.outlines[o];
                        bool building = record.building != 0;
                        Crossing cr;
                        cr.t = t;
                        cr.height_m = record.height_m;
                        cr.building = building;
                        cr.bounds_roof = building && edge_bounds_roof(s, start, delta, edge, record.first_vertex,
                                                                      record.vertex_count);
                        cr.footprint_id = record.footprint_id;
                        cr.edge = edge;
                        out.push_back(cr);
                    }
                }
            }
        }
        if (cell[0] == last[0] && cell[1] == last[1]) break;
        t_enter = std::min(t_max[0], t_max[1]);
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
    sort_and_deduplicate(out);
}

// The terrain at a position (steps): bilinear between the four DEM nodes around it, clamped to
// the DEM, as a terrain sample is read at a ray's ends (popup/src/scene.rs:182-200). A lattice
// point's differences are exact in f64, so it reads as its integer form did.
void terrain_at(const Scene &s, double x, double y, double &z, double &g) {
    if (s.dem_nx == 0) {
        z = s.flat_z;
        g = s.flat_g;
        return;
    }
    double fx = (x - (double)s.dem_ox) / (double)s.dem_spacing;
    double fy = (y - (double)s.dem_oy) / (double)s.dem_spacing;
    fx = std::min(std::max(fx, 0.0), (double)(s.dem_nx - 1));
    fy = std::min(std::max(fy, 0.0), (double)(s.dem_ny - 1));
    int64_t i0 = std::min<int64_t>((int64_t)std::floor(fx), s.dem_nx - 2);
    int64_t j0 = std::min<int64_t>((int64_t)std::floor(fy), s.dem_ny - 2);
    double ax = fx - i0, ay = fy - j0;
    auto node = [&](const std::vector<float> &v, int64_t i, int64_t j) { return (double)v[j * s.dem_nx + i]; };
    auto bil = [&](const std::vector<float> &v) {
        double lo = node(v, i0, j0) + ax * (node(v, i0 + 1, j0) - node(v, i0, j0));
        double hi = node(v, i0, j0 + 1) + ax * (node(v, i0 + 1, j0 + 1) - node(v, i0, j0 + 1));
        return lo + ay * (hi - lo);
    };
    z = bil(s.dem_z);
    g = bil(s.dem_g);
}

void terrain_at_point(const Scene &s, int64_t x, int64_t y, double &z, double &g) {
    terrain_at(s, (double)x, (double)y, z, g);
}

// The ground under a ray (popup/src/scene.rs:242-296 and walk :330-420, on one metric lattice):
// both ends, and a vertex wherever the ray crosses a row or a column line of the DEM strictly
// between them, in order; at a tie the row vertex comes first, then the column's at the same t.
void fill_profile(const Scene &s, const double from[2], const double to[2], Profile &profile) {
    double ox = (from[0] - to[0]) * s.step_m, oy = (from[1] - to[1]) * s.step_m;
    double length_m = std::hypot(ox, oy);
    profile.clear(std::max(length_m, 1.0));
    double z, g;
    terrain_at(s, from[0], from[1], z, g);
    profile.push(0.0, z, g);
    if (s.dem_nx != 0) {
        double sx = from[0], sy = from[1];
        double dx = to[0] - from[0], dy = to[1] - from[1];
        double sp = (double)s.dem_spacing;
        // Lattice line indices relative to the DEM origin.
        double cx = (sx - s.dem_ox) / sp, cy = (sy - s.dem_oy) / sp;
        double next_col = dx > 0 ? std::floor(cx) + 1.0 : std::ceil(cx) - 1.0;
        double next_row = dy > 0 ? std::floor(cy) + 1.0 : std::ceil(cy) - 1.0;
        double col_step = dx > 0 ? 1.0 : -1.0, row_step = dy > 0 ? 1.0 : -1.0;
        auto node = [&](const std::vector<float> &v, int64_t i, int64_t j) {
            i = std::min<int64_t>(std::max<int64_t>(i, 0), s.dem_nx - 1);
            j = std::min<int64_t>(std::max<int64_t>(j, 0), s.dem_ny - 1);
            return (double)v[j * s.dem_nx + i];
        };
        for (;;) {
            double t_col = dx != 0.0 ? (s.dem_ox + next_col * sp - sx) / dx : INF;
            double t_row = dy != 0.0 ? (s.dem_oy + next_row * sp - sy) / dy : INF;
            double t = std::min(t_col, t_row);
            if (t >= 1.0) break;
            double px = sx + t * dx, py = sy + t * dy;
            if (t_row <= t_col) {
                // On row line j = next_row: between nodes (i0, j) and (i0 + 1, j).
                double fx = (px - s.dem_ox) / sp;
                double i0 = std::floor(fx);
                double f = fx - i0;
                int64_t j = (int64_t)next_row, i = (int64_t)i0;
                double zz = node(s.dem_z, i, j) + f * (node(s.dem_z, i + 1, j) - node(s.dem_z, i, j));
                double gg = node(s.dem_g, i, j) + f * (node(s.dem_g, i + 1, j) - node(s.dem_g, i, j));
                profile.push(t, zz, gg);
                next_row += row_step;
            } else {
                double fy = (py - s.dem_oy) / sp;
                double j0 = std::floor(fy);
                double f = std::min(std::max(fy - j0, 0.0), 1.0);
                int64_t i = (int64_t)next_col, j = (int64_t)j0;
                double zz = node(s.dem_z, i, j) + f * (node(s.dem_z, i, j + 1) - node(s.dem_z, i, j));
                double gg = node(s.dem_g, i, j) + f * (node(s.dem_g, i, j + 1) - node(s.dem_g, i, j));
                profile.push(t, zz, gg);
                next_col += col_step;
            }
        }
    }
    terrain_at(s, to[0], to[1], z, g);
    profile.push(1.0, z, g);
}

// Whether lattice point (x, y) lies inside the closed ring of outline o (even-odd, exact).
bool point_in_ring(const Scene &s, const qm_outline &o, int64_t x, int64_t y) {
    bool inside = false;
    for (uint32_t k = 0; k + 1 < o.vertex_count; ++k) {
        uint32_t e = o.first_vertex + k;
        int64_t ax = s.vertices[2 * e], ay = s.vertices[2 * e + 1];
        int64_t bx = s.vertices[2 * e + 2], by = s.vertices[2 * e + 3];
        if ((ay > y) != (by > y)) {
            // x < ax + (y - ay) (bx - ax) / (by - ay), exactly.
            int64_t lhs = (x - ax) * (by - ay), rhs = (y - ay) * (bx - ax);
            if (by - ay > 0 ? lhs < rhs : lhs > rhs) inside = !inside;
        }
    }
    return inside;
}

// The building a point stands in, the lowest footprint id among those containing it (0 none),
// as `Point::at` finds it (paint/src/exact.rs:45-49).
uint64_t enclosing_building(const Scene &s, int64_t x, int64_t y) {
    uint64_t best = 0;
    for (const qm_outline &o : s.outlines) {
        if (!o.building || o.vertex_count < 4) continue;
        if (point_in_ring(s, o, x, y) && (best == 0 || o.footprint_id < best)) best = o.footprint_id;
    }
    return best;
}

Scene *scene_from_desc(const qm_scene_desc *d) {
    Scene *s = new Scene();
    s->step_m = d->step_m;
    s->cell_steps = d->cell_steps;
    s->cells_x = (d->extent_steps[0] + d->cell_steps - 1) / d->cell_steps;
    s->cells_y = (d->extent_steps[1] + d->cell_steps - 1) / d->cell_steps;
    s->vertices.assign(d->vertices, d->vertices + 2 * (size_t)d->n_vertices);
    s->outlines.assign(d->outlines, d->outlines + d->n_outlines);
    build_cells(*s);
    s->dem_nx = d->dem_nx;
    s->dem_ny = d->dem_ny;
    s->dem_ox = d->dem_origin[0];
    s->dem_oy = d->dem_origin[1];
    s->dem_spacing = d->dem_spacing;
    if (d->dem_nx) {
        s->dem_z.assign(d->dem_altitude_m, d->dem_altitude_m + (size_t)d->dem_nx * d->dem_ny);
        s->dem_g.assign(d->dem_ground_factor, d->dem_ground_factor + (size_t)d->dem_nx * d->dem_ny);
    }
    s->flat_z = d->flat_altitude_m;
    s->flat_g = d->flat_ground_factor;
    s->sources.assign(d->sources, d->sources + d->n_sources);
    std::memcpy(s->favourable, d->favourable, sizeof(s->favourable));
    for (int b = 0; b < BANDS; ++b) s->alpha[b] = d->alpha_db_per_km[b];
    return s;
}

struct Receiver {
    int64_t x, y;
    double altitude_m;
    uint64_t own_footprint;
};

struct PairResult {
    double bands[PERIODS][BANDS];  // received energy per period and band
    double states[2][PERIODS];     // path.states
};

struct Worker {
    Profile profile;
    std::vector<Crossing> crossings;
    RayScratch ray;
};

// The walks from and to lattice points (exact in f64, so these read as the f64 forms do).
void scene_crossings(const Scene &s, const int64_t from[2], const int64_t to[2], std::vector<Crossing> &out,
                     uint64_t *edges_tested = nullptr) {
    const double f[2] = {(double)from[0], (double)from[1]}, t[2] = {(double)to[0], (double)to[1]};
    scene_crossings(s, f, t, out, edges_tested);
}

void fill_profile(const Scene &s, const int64_t from[2], const int64_t to[2], Profile &profile) {
    const double f[2] = {(double)from[0], (double)from[1]}, t[2] = {(double)to[0], (double)to[1]};
    fill_profile(s, f, t, profile);
}

// One point source at one receiver: `source_rays` for a point and `add_ray`
// (popup/src/evaluate.rs:119-152, 171-214, 300-330), `whole_energy` (paint/src/exact.rs:186-205).
void evaluate_pair(const Scene &s, const Receiver &r, const qm_source &src, Worker &w, PairResult &out,
                   bool want_favourable = true, uint64_t *edges_tested = nullptr) {
    int64_t from[2] = {src.x, src.y}, to[2] = {r.x, r.y};
    fill_profile(s, from, to, w.profile);
    scene_crossings(s, from, to, w.crossings, edges_tested);
    if (r.own_footprint != 0) {
        size_t kept = 0;
        for (size_t i = 0; i < w.crossings.size(); ++i)
            if (w.crossings[i].footprint_id != r.own_footprint) w.crossings[kept++] = w.crossings[i];
        w.crossings.resize(kept);
    }
    double azimuth = std::atan2((double)(r.y - src.y) * s.step_m, (double)(r.x - src.x) * s.step_m);
    double p[PERIODS];
    for (int period = 0; period < PERIODS; ++period) p[period] = favourable_at(s.favourable[period], azimuth);
    RayEnds ends;
    ends.source_height_m = src.height_m;
    ends.has_source_ground = false;
    ends.source_ground_m = 0.0;
    ends.receiver_altitude_m = r.altitude_m;
    ends.has_source_ground_factor = src.ground_factor >= 0.0f;
    ends.source_ground_factor = src.ground_factor;
    ends.platform_half_width_m = src.platform_half_width_m;
    ends.own_footprint = src.footprint_id;
    Transfer transfer;
    StateBoundary boundaries[2];
    ray_terms(w.profile, w.crossings, ends, p, s.alpha, w.ray, transfer, boundaries, want_favourable);
    double dh = std::hypot((double)(src.x - r.x) * s.step_m, (double)(src.y - r.y) * s.step_m);
    double ground0 = w.profile.ground_m[0];
    double distance =
        std::max(std::hypot(std::max(dh, (double)src.exclusion_radius_m), r.altitude_m - (ground0 + src.height_m)), 1.0);
    double weight = 1.0 / (distance * distance * energy(11.0));
    for (int period = 0; period < PERIODS; ++period) {
        for (int st = 0; st < 2; ++st) out.states[st][period] = 0.0;
        for (int b = 0; b < BANDS; ++b) {
            double power = weight * (double)src.energy[period][b];
            out.bands[period][b] = power * transfer.periods[period][b];
            out.states[0][period] += power * transfer.states[0][b];
            out.states[1][period] += power * transfer.states[1][b];
        }
    }
}

Receiver make_receiver(const Scene &s, int64_t x, int64_t y, double height_m, uint64_t own) {
    double z, g;
    terrain_at_point(s, x, y, z, g);
    return Receiver{x, y, z + height_m, own};
}

bool favourable_needed(const Scene &s) {
    for (int p = 0; p < PERIODS; ++p)
        for (int k = 0; k < SECTORS; ++k)
            if (s.favourable[p][k] != 0.0f) return true;
    return false;
}

template <class F>
void parallel_for(size_t n, int threads, F f) {
    if (threads <= 1 || n < 2) {
        for (size_t i = 0; i < n; ++i) f(i, 0);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i, t);
            }
        });
    for (auto &th : pool) th.join();
}

// ---------------------------------------------------------------------------------------------
// ISO 532-1 Zwicker loudness: physics/src/loudness.rs:11-182
const double RAP[8] = {45.0, 55.0, 65.0, 71.0, 80.0, 90.0, 100.0, 120.0};
const double DLL[8][11] = {
    {-32.0, -24.0, -16.0, -10.0, -5.0, 0.0, -7.0, -3.0, 0.0, -2.0, 0.0},
    {-29.0, -22.0, -15.0, -10.0, -4.0, 0.0, -7.0, -2.0, 0.0, -2.0, 0.0},
    {-27.0, -19.0, -14.0, -9.0, -4.0, 0.0, -6.0, -2.0, 0.0, -2.0, 0.0},
    {-25.0, -17.0, -12.0, -9.0, -3.0, 0.0, -5.0, -2.0, 0.0, -2.0, 0.0},
    {-23.0, -16.0, -11.0, -7.0, -3.0, 0.0, -4.0, -1.0, 0.0, -1.0, 0.0},
    {-20.0, -14.0, -10.0, -6.0, -3.0, 0.0, -4.0, -1.0, 0.0, -1.0, 0.0},
    {-18.0, -12.0, -9.0, -6.0, -2.0, 0.0, -3.0, -1.0, 0.0, -1.0, 0.0},
    {-15.0, -10.0, -8.0, -4.0, -2.0, 0.0, -3.0, -1.0, 0.0, -1.0, 0.0},
};
const double LTQ[20] = {30.0, 18.0, 12.0, 8.0, 7.0, 6.0, 5.0, 4.0, 3.0, 3.0,
                        3.0, 3.0, 3.0, 3.0, 3.0, 3.0, 3.0, 3.0, 3.0, 3.0};
const double A0[20] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0,
                       -0.5, -1.6, -3.2, -5.4, -5.6, -4.0, -1.5, 2.0, 5.0, 12.0};
const double DCB[20] = {-0.25, -0.6, -0.8, -0.8, -0.5, 0.0, 0.5, 1.1, 1.5, 1.7,
                        1.8, 1.8, 1.7, 1.6, 1.4, 1.2, 0.8, 0.5, 0.0, -0.5};
const double ZUP[21] = {0.9, 1.8, 2.8, 3.5, 4.4, 5.4, 6.6, 7.9, 9.2, 10.6, 12.3,
                        13.8, 15.2, 16.7, 18.1, 19.3, 20.6, 21.8, 22.7, 23.6, 24.0};
const double RNS[18] = {21.5, 18.0, 15.1, 11.5, 9.0, 6.1, 4.4, 3.1, 2.13,
                        1.36, 0.82, 0.42, 0.30, 0.22, 0.15, 0.10, 0.035, 0.0};
const double USL[18][8] = {
    {13.0, 8.2, 6.3, 5.5, 5.5, 5.5, 5.5, 5.5},       {9.0, 7.5, 6.0, 5.1, 4.5, 4.5, 4.5, 4.5},
    {7.8, 6.7, 5.6, 4.9, 4.4, 3.9, 3.9, 3.9},        {6.2, 5.4, 4.6, 4.0, 3.5, 3.2, 3.2, 3.2},
    {4.5, 3.8, 3.6, 3.2, 2.9, 2.7, 2.7, 2.7},        {3.7, 3.0, 2.8, 2.35, 2.2, 2.2, 2.2, 2.2},
    {2.9, 2.3, 2.1, 1.9, 1.8, 1.7, 1.7, 1.7},        {2.4, 1.7, 1.5, 1.35, 1.3, 1.3, 1.3, 1.3},
    {1.95, 1.45, 1.3, 1.15, 1.1, 1.1, 1.1, 1.1},     {1.5, 1.2, 0.94, 0.86, 0.82, 0.82, 0.82, 0.82},
    {0.72, 0.67, 0.64, 0.63, 0.62, 0.62, 0.62, 0.62}, {0.59, 0.53, 0.51, 0.50, 0.42, 0.42, 0.42, 0.42},
    {0.40, 0.33, 0.26, 0.24, 0.24, 0.22, 0.22, 0.22}, {0.27, 0.21, 0.20, 0.18, 0.17, 0.17, 0.17, 0.17},
    {0.16, 0.15, 0.14, 0.12, 0.11, 0.11, 0.11, 0.11}, {0.12, 0.11, 0.10, 0.08, 0.08, 0.08, 0.08, 0.08},
    {0.09, 0.08, 0.07, 0.06, 0.06, 0.06, 0.06, 0.05}, {0.06, 0.05, 0.03, 0.02, 0.02, 0.02, 0.02, 0.02},
};

// loudness.rs:100-144
void core_loudness(const double levels[28], double core[21]) {
    double corrected[11];
    for (int band = 0; band < 11; ++band) {
        double level = levels[band];
        int range = 7;
        for (int k = 0; k < 8; ++k)
            if (level <= RAP[k] - DLL[k][band]) {
                range = k;
                break;
            }
        corrected[band] = energy(level + DLL[range][band]);
    }
    double lowest[3];
    const int lo[3] = {0, 6, 9}, hi[3] = {6, 9, 11};
    for (int k = 0; k < 3; ++k) {
        double sum = 0.0;
        for (int b = lo[k]; b < hi[k]; ++b) sum += corrected[b];
        lowest[k] = sum > 0.0 ? 10.0 * std::log10(sum) : -INF;
    }
    for (int b = 0; b < 21; ++b) core[b] = 0.0;
    for (int band = 0; band < 20; ++band) {
        double level = (band < 3 ? lowest[band] : levels[band + 8]) - A0[band];
        if (level > LTQ[band]) {
            level -= DCB[band];
            double s = 0.25;
            double threshold = energy(LTQ[band] / 4.0);
            core[band] = std::max(0.0635 * threshold *
                                      (std::sqrt(std::sqrt(1.0 - s + s * energy(level - LTQ[band]))) - 1.0),
                                  0.0);
        }
    }
    double correction = 0.4 + 0.32 * std::pow(core[0], 0.2);
    if (correction <= 1.0) core[0] *= correction;
}

// loudness.rs:148-182
double zwicker_loudness_sone(const double in_levels[28]) {
    double levels[28];
    for (int i = 0; i < 28; ++i) levels[i] = std::max(in_levels[i], -60.0);
    double core[21];
    core_loudness(levels, core);
    double total = 0.0, z1 = 0.0, n1 = 0.0;
    for (int band = 0; band < 21; ++band) {
        double upper = ZUP[band] + 0.0001;
        int group = std::min(std::max(band - 1, 0), 7);
        double c = core[band];
        while (z1 < upper) {
            if (n1 <= c) {
                total += c * (upper - z1);
                z1 = upper;
                n1 = c;
            } else {
                int range = 17;
                for (int k = 0; k < 18; ++k)
                    if (n1 > RNS[k]) {
                        range = k;
                        break;
                    }
                double steepness = USL[range][group];
                double n2 = std::max(RNS[range], c);
                double z2 = z1 + (n1 - n2) / steepness;
                if (z2 > upper) {
                    z2 = upper;
                    n2 = n1 - (z2 - z1) * steepness;
                }
                total += (z2 - z1) * (n1 + n2) / 2.0;
                z1 = z2;
                n1 = n2;
            }
        }
    }
    return std::max(total, 0.0);
}

// popup/src/distribution.rs:69-72 with Rust's saturating float-to-usize cast.
uint32_t level_bin(double level_db, double level_min, double bin_db, uint32_t n_bins) {
    double r = std::round((level_db - level_min) / bin_db);
    uint64_t k;
    if (!(r > 0.0))
        k = 0;  // negative and NaN saturate to 0
    else if (r >= 1.8446744073709552e19)
        k = UINT64_MAX;
    else
        k = (uint64_t)r;
    return (uint32_t)std::min<uint64_t>(k, n_bins - 1);
}

}  // namespace

// =============================================================================================
// C entry points (ctypes).
// The terrain feature set of include/qm_surrogate.h for one path, two rows (homogeneous and
// favourable): 3 DEM samples in each of 12 stretches (ends at 0, 2, 5, 10, 20, 35, 50, 65, 80, 90,
// 95, 98, 100 % of the path) at lattice points rounded from t along the path, the largest rise
// of the ground above the straight source-receiver line in each stretch,
// and the largest rise of the obstacle tops crossed (walls standing on the ground at their
// rounded crossing points) in each stretch.
void terrain_sample(const Scene &s, const qm_source &src, const Receiver &r, const Worker &w, const PathBuffers &pb,
                    const StateBoundary boundaries[2], double *f, double *labels, uint8_t *eligible) {
    const int64_t dx = r.x - src.x, dy = r.y - src.y;
    const double L = std::max(w.profile.horizontal_m, 1.0);
    double zs, gs, zr, gr;
    terrain_at_point(s, src.x, src.y, zs, gs);
    terrain_at_point(s, r.x, r.y, zr, gr);
    const double src_alt = zs + src.height_m;
    const double rise = (r.altitude_m - src_alt) / L;
    auto ground_at = [&](double t, double &z, double &g) {
        int64_t px = src.x + (int64_t)std::llrint(t * (double)dx), py = src.y + (int64_t)std::llrint(t * (double)dy);
        terrain_at_point(s, px, py, z, g);
    };
    const float E[13] = {0.0f, 0.02f, 0.05f, 0.1f, 0.2f, 0.35f, 0.5f, 0.65f, 0.8f, 0.9f, 0.95f, 0.98f, 1.0f};
    double gsum = 0.0;
    for (int j = 0; j < 12; ++j) {
        double top = -INF;
        for (int q = 0; q < 3; ++q) {
            double t = (double)E[j] + (q + 0.5) / 3.0 * (double)(E[j + 1] - E[j]), z, g;
            ground_at(t, z, g);
            top = std::max(top, z - (src_alt + rise * t * L));
            gsum += g;
        }
        f[8 + j] = top / 10.0;
    }
    for (int j = 0; j < 12; ++j) f[20 + j] = -10.0;
    for (const Crossing &c : w.crossings) {
        if (std::binary_search(pb.containing.begin(), pb.containing.end(), c.footprint_id)) continue;
        double z, g;
        ground_at(c.t, z, g);
        int j = 0;
        while (j < 11 && c.t >= (double)E[j + 1]) ++j;
        f[20 + j] = std::max(f[20 + j], (z + c.height_m - (src_alt + rise * c.t * L)) / 10.0);
    }
    const bool ok = true;
    f[0] = L / 1000.0;
    f[1] = src.height_m / 10.0;
    f[2] = (r.altitude_m - zr) / 10.0;
    f[3] = (zr - zs) / 10.0;
    f[5] = src.ground_factor >= 0.0f ? (double)src.ground_factor : gs;
    f[6] = gsum / 36.0;
    f[7] = gr;
    for (int state = 0; state < 2; ++state) {
        double *fs = f + state * 32;
        if (state == 1)
            for (int k = 0; k < 32; ++k) fs[k] = f[k];
        fs[4] = (double)state;
        for (int b = 0; b < BANDS; ++b) labels[state * BANDS + b] = boundaries[state].attenuation[b];
        eligible[state] = ok ? 1 : 0;
    }
}

extern "C" {

int qmo_version(void) { return 1; }

void qmo_alpha_bands(double temperature_c, double rh, double out[8]) {
    for (int b = 0; b < BANDS; ++b)
        out[b] = alpha_db_per_km(exact_mid_band_frequency_hz(b), temperature_c, rh, 101.325);
}

// A_boundary of both states of one vertical path (physics/src/cnossos/mod.rs:123), for the
// ISO/TR 17534-4 acceptance test: out_attenuation[2][8], out_without_ground[2][8].
void qmo_state_boundaries(const double *d, const double *z, const double *g, size_t n, double sx, double sz,
                          double rx, double rz, double source_ground_factor, const double *terrain_xz,
                          size_t n_terrain, const double *tops_xz, size_t n_tops, double *out_attenuation,
                          double *out_without_ground) {
    VPath path;
    path.profile = VProfile{d, z, g, n};
    path.source = PP{sx, sz};
    path.receiver = PP{rx, rz};
    path.source_ground_factor = source_ground_factor;
    std::vector<PP> terrain(n_terrain), tops(n_tops);
    for (size_t i = 0; i < n_terrain; ++i) terrain[i] = PP{terrain_xz[2 * i], terrain_xz[2 * i + 1]};
    for (size_t i = 0; i < n_tops; ++i) tops[i] = PP{tops_xz[2 * i], tops_xz[2 * i + 1]};
    path.terrain = terrain.data();
    path.n_terrain = n_terrain;
    path.tops = tops.data();
    path.n_tops = n_tops;
    PathScratch s;
    StateBoundary out[2];
    state_boundaries(path, s, out, true);
    for (int st = 0; st < 2; ++st)
        for (int b = 0; b < BANDS; ++b) {
            out_attenuation[st * BANDS + b] = out[st].attenuation[b];
            out_without_ground[st * BANDS + b] = out[st].without_ground[b];
        }
}

// One ray's transfer (physics/src/ray.rs:125): crossings as rows of (t, height, building,
// bounds_roof, footprint). Outputs slant, periods[3][8], states[2][8], and the vertical path
// it built (path_d/z/g with capacity `cap`, n_path) and its obstacle tops (tops_xz, n_tops).
void qmo_ray_terms(double horizontal_m, const double *t, const double *ground_m, const double *ground_factor,
                   size_t n_profile, const double *crossing_t, const double *crossing_height,
                   const int32_t *crossing_building, const int32_t *crossing_bounds, const uint64_t *crossing_fp,
                   size_t n_crossings, double source_height_m, int has_source_ground, double source_ground_m,
                   double receiver_altitude_m, int has_source_gf, double source_gf, double platform_half_width_m,
                   uint64_t own_footprint, const double p[3], const double alpha[8], double *out_slant,
                   double *out_periods, double *out_states, double *path_d, double *path_z, double *path_g,
                   size_t cap, size_t *n_path, double *tops_xz, size_t tops_cap, size_t *n_tops) {
    Profile profile;
    profile.clear(horizontal_m);
    for (size_t i = 0; i < n_profile; ++i) profile.push(t[i], ground_m[i], ground_factor[i]);
    std::vector<Crossing> crossings(n_crossings);
    for (size_t i = 0; i < n_crossings; ++i)
        crossings[i] = Crossing{crossing_t[i], crossing_height[i], crossing_building[i] != 0, crossing_bounds[i] != 0,
                                crossing_fp[i], 0};
    RayEnds ends{source_height_m,  has_source_ground != 0, source_ground_m,       receiver_altitude_m,
                 has_source_gf != 0, source_gf,            platform_half_width_m, own_footprint};
    RayScratch scratch;
    Transfer transfer;
    StateBoundary b[2];
    ray_terms(profile, crossings, ends, p, alpha, scratch, transfer, b, true);
    *out_slant = transfer.slant_m;
    for (int period = 0; period < PERIODS; ++period)
        for (int band = 0; band < BANDS; ++band) out_periods[period * BANDS + band] = transfer.periods[period][band];
    for (int st = 0; st < 2; ++st)
        for (int band = 0; band < BANDS; ++band) out_states[st * BANDS + band] = transfer.states[st][band];
    // The path as built (fill again: ray_terms left it in scratch).
    const PathBuffers &pb = scratch.pb;
    *n_path = pb.d.size();
    for (size_t i = 0; i < pb.d.size() && i < cap; ++i) {
        path_d[i] = pb.d[i];
        path_z[i] = pb.z[i];
        path_g[i] = pb.g[i];
    }
    *n_tops = pb.tops.size();
    for (size_t i = 0; i < pb.tops.size() && i < tops_cap; ++i) {
        tops_xz[2 * i] = pb.tops[i].x;
        tops_xz[2 * i + 1] = pb.tops[i].z;
    }
}

// The crests of a terrain polyline (physics/src/ray.rs:360): out_xz capacity `cap`.
size_t qmo_crests_of(const double *xz, size_t n, double length, double *out_xz, size_t cap) {
    std::vector<PP> terrain(n), out;
    for (size_t i = 0; i < n; ++i) terrain[i] = PP{xz[2 * i], xz[2 * i + 1]};
    crests_of(terrain, length, out);
    for (size_t i = 0; i < out.size() && i < cap; ++i) {
        out_xz[2 * i] = out[i].x;
        out_xz[2 * i + 1] = out[i].z;
    }
    return out.size();
}

void *qmo_scene_new(const qm_scene_desc *desc) { return scene_from_desc(desc); }
void qmo_scene_free(void *scene) { delete static_cast<Scene *>(scene); }

// Crossings of the ray from -> to (lattice steps): rows of t (f64), and per crossing its
// footprint id, edge start vertex, bounds_roof and building. Returns the count (capped writes).
size_t qmo_crossings(void *scene, const int64_t from[2], const int64_t to[2], double *t, uint64_t *footprint,
                     uint32_t *edge, int32_t *bounds_roof, int32_t *building, size_t cap) {
    const Scene &s = *static_cast<Scene *>(scene);
    std::vector<Crossing> out;
    scene_crossings(s, from, to, out);
    for (size_t i = 0; i < out.size() && i < cap; ++i) {
        t[i] = out[i].t;
        footprint[i] = out[i].footprint_id;
        edge[i] = out[i].edge;
        bounds_roof[i] = out[i].bounds_roof;
        building[i] = out[i].building;
    }
    return out.size();
}

// The same for ends anywhere (f64 steps), as the reference's walk takes them off the lattice
// (popup/src/obstacles/mod.rs:61-73).
size_t qmo_crossings_d(void *scene, const double from[2], const double to[2], double *t, uint64_t *footprint,
                       uint32_t *edge, int32_t *bounds_roof, int32_t *building, size_t cap) {
    const Scene &s = *static_cast<Scene *>(scene);
    std::vector<Crossing> out;
    scene_crossings(s, from, to, out);
    for (size_t i = 0; i < out.size() && i < cap; ++i) {
        t[i] = out[i].t;
        footprint[i] = out[i].footprint_id;
        edge[i] = out[i].edge;
        bounds_roof[i] = out[i].bounds_roof;
        building[i] = out[i].building;
    }
    return out.size();
}

// Every edge of every outline against the ray, with the walk's deduplication: the list the walk
// must give (the reference's own check of its walk, popup/src/obstacles/tests/mod.rs:198-229).
size_t qmo_crossings_every(void *scene, const double from[2], const double to[2], double *t, uint64_t *footprint,
                           uint32_t *edge, int32_t *bounds_roof, int32_t *building, size_t cap) {
    const Scene &s = *static_cast<Scene *>(scene);
    const double start[2] = {from[0], from[1]}, delta[2] = {to[0] - from[0], to[1] - from[1]};
    std::vector<Crossing> out;
    for (size_t o = 0; o < s.outlines.size(); ++o) {
        const qm_outline &record = s.outlines[o];
        for (uint32_t k = 0; k + 1 < record.vertex_count; ++k) {
            const size_t e = record.first_vertex + k;
            const double a[2] = {(double)s.vertices[2 * e], (double)s.vertices[2 * e + 1]};
            const double b[2] = {(double)s.vertices[2 * e + 2], (double)s.vertices[2 * e + 3]};
            double tt;
            if (!segment_intersection_t(start, delta, a, b, tt)) continue;
            Crossing cr;
            cr.t = tt;
            cr.height_m = record.height_m;
            cr.building = record.building != 0;
            cr.bounds_roof = cr.building && edge_bounds_roof(s, start, delta, e, record.first_vertex, record.vertex_count);
            cr.footprint_id = record.footprint_id;
            cr.edge = (uint32_t)e;
            out.push_back(cr);
        }
    }
    sort_and_deduplicate(out);
    for (size_t i = 0; i < out.size() && i < cap; ++i) {
        t[i] = out[i].t;
        footprint[i] = out[i].footprint_id;
        edge[i] = out[i].edge;
        bounds_roof[i] = out[i].bounds_roof;
        building[i] = out[i].building;
    }
    return out.size();
}

// The building enclosing each of n lattice points (0 none).
void qmo_enclosing_buildings(void *scene, const int64_t *xy, size_t n, uint64_t *out, int threads) {
    const Scene &s = *static_cast<Scene *>(scene);
    parallel_for(n, threads, [&](size_t i, int) { out[i] = enclosing_building(s, xy[2 * i], xy[2 * i + 1]); });
}

// The ground profile under a ray (altitude and G at t): returns the count, capped writes.
size_t qmo_profile(void *scene, const int64_t from[2], const int64_t to[2], double *t, double *z, double *g,
                   size_t cap, double *horizontal_m) {
    const Scene &s = *static_cast<Scene *>(scene);
    Profile p;
    fill_profile(s, from, to, p);
    *horizontal_m = p.horizontal_m;
    for (size_t i = 0; i < p.t.size() && i < cap; ++i) {
        t[i] = p.t[i];
        z[i] = p.ground_m[i];
        g[i] = p.ground_factor[i];
    }
    return p.t.size();
}

// The ground profile under a ray with ends anywhere (f64 steps).
size_t qmo_profile_d(void *scene, const double from[2], const double to[2], double *t, double *z, double *g,
                     size_t cap, double *horizontal_m) {
    const Scene &s = *static_cast<Scene *>(scene);
    Profile p;
    fill_profile(s, from, to, p);
    *horizontal_m = p.horizontal_m;
    for (size_t i = 0; i < p.t.size() && i < cap; ++i) {
        t[i] = p.t[i];
        z[i] = p.ground_m[i];
        g[i] = p.ground_factor[i];
    }
    return p.t.size();
}

// Batch::evaluate over pairs (paint/src/exact.rs:218-254): receivers as lattice points with
// altitude (absolute m), own footprint and point; pairs (source, receiver, band weight).
// Outputs pair_sums[n][9] (mixed[3], calm[3], downwind[3]), pair_bands[n][3][8] (nullable),
// point_bands[n_points][6][3][8] (accumulated in pair order).
void qmo_evaluate_pairs(void *scene, const int64_t *receiver_xy, const double *receiver_altitude,
                        const uint64_t *own_footprint, const uint32_t *point_of_receiver, size_t n_receivers,
                        const uint32_t *source_of_pair, const uint32_t *receiver_of_pair, const double *band_weight,
                        size_t n_pairs, double *pair_sums, double *pair_bands, double *point_bands, size_t n_points,
                        int threads) {
    (void)n_receivers;
    (void)n_points;
    const Scene &s = *static_cast<Scene *>(scene);
    std::vector<PairResult> results(n_pairs);
    std::vector<Worker> workers(std::max(threads, 1));
    parallel_for(n_pairs, threads, [&](size_t i, int t) {
        uint32_t r = receiver_of_pair[i];
        Receiver rec{receiver_xy[2 * r], receiver_xy[2 * r + 1], receiver_altitude[r], own_footprint[r]};
        evaluate_pair(s, rec, s.sources[source_of_pair[i]], workers[t], results[i], true);
    });
    for (size_t i = 0; i < n_pairs; ++i) {
        const PairResult &pr = results[i];
        for (int period = 0; period < PERIODS; ++period) {
            double mixed = 0.0;
            for (int b = 0; b < BANDS; ++b) mixed += pr.bands[period][b];
            pair_sums[i * 9 + period] = mixed;
            pair_sums[i * 9 + 3 + period] = pr.states[0][period];
            pair_sums[i * 9 + 6 + period] = pr.states[1][period];
        }
        if (pair_bands)
            for (int period = 0; period < PERIODS; ++period)
                for (int b = 0; b < BANDS; ++b) pair_bands[(i * PERIODS + period) * BANDS + b] = pr.bands[period][b];
        uint32_t point = point_of_receiver[receiver_of_pair[i]];
        uint32_t layer = s.sources[source_of_pair[i]].layer;
        double w = band_weight ? band_weight[i] : 1.0;
        for (int period = 0; period < PERIODS; ++period)
            for (int b = 0; b < BANDS; ++b)
                point_bands[((size_t)point * QM_LAYERS * PERIODS + layer * PERIODS + period) * BANDS + b] +=
                    w * pr.bands[period][b];
    }
}

// The grid painter (evaluate_all over a regular grid of receivers): per cell the day band
// energies (out_energy[cells][8]) and the Lden-weighted A energy (out_lden_energy[cells]), summed
// over sources [begin, end). Cells [cell_begin, cell_end) only (a sample), or all when equal.
// Returns the number of edge box tests in *edges_tested (the crossing walk's work).
void qmo_paint_grid(void *scene, const qm_grid_desc *grid, uint32_t cell_begin, uint32_t cell_end,
                    double *out_energy, double *out_lden_energy, int threads, uint64_t *edges_tested) {
    const Scene &s = *static_cast<Scene *>(scene);
    uint32_t n_cells = (uint32_t)(grid->nx * grid->ny);
    if (cell_end <= cell_begin) {
        cell_begin = 0;
        cell_end = n_cells;
    }
    uint32_t sb = grid->source_begin, se = grid->source_end;
    if (se <= sb) {
        sb = 0;
        se = (uint32_t)s.sources.size();
    }
    bool fav = favourable_needed(s);
    std::vector<Worker> workers(std::max(threads, 1));
    std::vector<uint64_t> tested(std::max(threads, 1), 0);
    double lden_w[PERIODS];
    for (int p = 0; p < PERIODS; ++p) lden_w[p] = PERIOD_HOURS[p] * energy(PERIOD_PENALTY_DB[p]) / 24.0;
    parallel_for(cell_end - cell_begin, threads, [&](size_t k, int t) {
        uint32_t cell = cell_begin + (uint32_t)k;
        int64_t x = grid->origin[0] + (int64_t)(cell % grid->nx) * grid->spacing;
        int64_t y = grid->origin[1] + (int64_t)(cell / grid->nx) * grid->spacing;
        Receiver r = make_receiver(s, x, y, grid->height_m, enclosing_building(s, x, y));
        double e[BANDS] = {0};
        double lden = 0.0;
        PairResult pr;
        for (uint32_t src = sb; src < se; ++src) {
            evaluate_pair(s, r, s.sources[src], workers[t], pr, fav, &tested[t]);
            for (int b = 0; b < BANDS; ++b) e[b] += pr.bands[0][b];
            for (int p = 0; p < PERIODS; ++p)
                for (int b = 0; b < BANDS; ++b) lden += lden_w[p] * pr.bands[p][b];
        }
        for (int b = 0; b < BANDS; ++b) out_energy[k * BANDS + b] = e[b];
        out_lden_energy[k] = lden;
    });
    if (edges_tested) {
        uint64_t total = 0;
        for (uint64_t v : tested) total += v;
        *edges_tested = total;
    }
}

// Work counts of one pair (for sizing device buffers): crossings, profile vertices, candidates,
// blocking candidates and hull points per state. out[7].
void qmo_path_counts(void *scene, const int64_t from[2], const int64_t to[2], double *out) {
    const Scene &s = *static_cast<Scene *>(scene);
    Worker w;
    fill_profile(s, from, to, w.profile);
    scene_crossings(s, from, to, w.crossings);
    RayEnds ends{0.05, false, 0.0, 0.0, false, 0.0, 0.0, 0};
    double z, g;
    terrain_at_point(s, to[0], to[1], z, g);
    ends.receiver_altitude_m = z + 4.0;
    fill_path(w.ray.pb, w.profile, w.crossings, ends);
    const PathBuffers &pb = w.ray.pb;
    VPath path;
    path.profile = VProfile{pb.d.data(), pb.z.data(), pb.g.data(), pb.d.size()};
    double length = pb.d.back();
    path.source = PP{0.0, w.profile.ground_m[0] + 0.05};
    path.receiver = PP{length, ends.receiver_altitude_m};
    path.source_ground_factor = w.profile.ground_factor[0];
    path.terrain = pb.crests.data();
    path.n_terrain = pb.crests.size();
    path.tops = pb.tops.data();
    path.n_tops = pb.tops.size();
    PathScratch ps;
    collect_candidates(path, ps.candidates);
    out[0] = (double)w.crossings.size();
    out[1] = (double)pb.d.size();
    out[2] = (double)ps.candidates.size();
    for (int st = 0; st < 2; ++st) {
        StateRay ray = StateRay::between(st, path.source, path.receiver);
        bool blocked;
        diffraction_path(ray, path.source, path.receiver, ps.candidates, ps.blocking, ps.hull, ps.points, blocked);
        out[3 + 2 * st] = (double)ps.blocking.size();
        out[4 + 2 * st] = blocked ? (double)ps.points.size() : 0.0;
    }
}

double qmo_zwicker(const double *levels28) { return zwicker_loudness_sone(levels28); }

void qmo_zwicker_many(const double *levels, size_t n, double *sone, int threads) {
    parallel_for(n, threads, [&](size_t i, int) { sone[i] = zwicker_loudness_sone(levels + 28 * i); });
}

void qmo_level_histogram(const double *levels, size_t n, double level_min, double bin_db, uint32_t n_bins,
                         uint32_t *counts) {
    for (uint32_t k = 0; k < n_bins; ++k) counts[k] = 0;
    for (size_t i = 0; i < n; ++i) counts[level_bin(levels[i], level_min, bin_db, n_bins)]++;
}

// ---------------------------------------------------------------------------------------------
// Line pieces: the CNOSSOS-EU point sum of a straight piece by quadrature in the in-plane angle
// (physics/src/line.rs). Positions are receiver-relative metres (x east, y north, z up).

static const double LINE_PI = 3.14159265358979323846;
static const int LINE_BUCKETS = 5;                                   // line.rs:19
static const double LINE_ONE_BUCKET_SPAN = 3.0 * LINE_PI / 180.0;    // line.rs:23
static const double LINE_WIDE_MIN_SPAN = 3.0 * LINE_PI / 180.0;      // line.rs:26
static const int LINE_MASK_BINS = 128;                               // line.rs:28
static const double LINE_PART_MAX_SPAN = 0.26;                       // line.rs:30
static const int LINE_MAX_PARTS = 9;                                 // line.rs:31
static const double LINE_PERP_FLOOR = 0.5;                           // line.rs:34
static const double LINE_DIVERGENCE = 12.589254117941673;            // 10^1.1, line.rs:36

static double line_wrap_to_pi(double angle) {  // line.rs:39-48
    const double tau = 2.0 * LINE_PI;
    double a = std::fmod(angle, tau);
    if (a > LINE_PI) return a - tau;
    if (a <= -LINE_PI) return a + tau;
    return a;
}

struct LinePiece {  // line.rs:53-62, 86-124
    double start[3], unit[3], length, foot, perp, angle0, angle1;
    bool make(const double s[3], const double e[3]) {
        const double a[3] = {e[0] - s[0], e[1] - s[1], e[2] - s[2]};
        length = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
        if (length < 1e-3) return false;
        for (int k = 0; k < 3; ++k) {
            start[k] = s[k];
            unit[k] = a[k] / length;
        }
        foot = -(s[0] * unit[0] + s[1] * unit[1] + s[2] * unit[2]);
        const double f[3] = {s[0] + foot * unit[0], s[1] + foot * unit[1], s[2] + foot * unit[2]};
        perp = std::max(std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]), LINE_PERP_FLOOR);
        angle0 = std::atan((0.0 - foot) / perp);
        angle1 = std::atan((length - foot) / perp);
        return true;
    }
    double span() const { return angle1 - angle0; }
    double divergence() const { return std::hypot(unit[0], unit[1]) / (LINE_DIVERGENCE * perp); }
    double angle_at(double along) const { return std::atan((along - foot) / perp); }
    double along_at_angle(double angle) const {
        return std::min(std::max(foot + perp * std::tan(angle), 0.0), length);
    }
    void point(double along, double p[3]) const {
        for (int k = 0; k < 3; ++k) p[k] = start[k] + along * unit[k];
    }
    // Where the horizontal ray at `azimuth` meets the ground track, clamped; false when parallel.
    bool along_at_azimuth(double azimuth, double &along) const {
        const double dx = std::cos(azimuth), dy = std::sin(azimuth);
        const double ux = unit[0] * length, uy = unit[1] * length;
        const double den = dx * uy - dy * ux;
        if (std::fabs(den) < 1e-12) return false;
        const double fraction = (dy * start[0] - dx * start[1]) / den;
        along = std::min(std::max(fraction, 0.0), 1.0) * length;
        return true;
    }
    double azimuth_at(double along) const {
        double p[3];
        point(along, p);
        return std::atan2(p[1], p[0]);
    }
    double range_at(double along) const {
        double p[3];
        point(along, p);
        return std::hypot(p[0], p[1]);
    }
};

struct LineNode {
    double along, weight;
    bool on_ray;
};

// mark_blocked_bins (line.rs:317-355): the bins of the span one edge's arc blocks where the edge
// stands at least a metre nearer than the piece seen there.
static void line_mark(const LinePiece &g, const double arc[3], double radius, double lo, double hi, double width,
                      bool blocked[LINE_MASK_BINS]) {
    if (arc[2] > radius) return;
    for (double shift : {0.0, 2.0 * LINE_PI, -2.0 * LINE_PI}) {
        const double piece_lo = std::max(arc[0] + shift, lo), piece_hi = std::min(arc[1] + shift, hi);
        if (piece_hi <= piece_lo) continue;
        double along;
        if (!g.along_at_azimuth(0.5 * (piece_lo + piece_hi), along)) continue;
        if (g.range_at(along) - arc[2] <= 1.0) continue;
        // A first bin past the end (an overlap rounded onto the span's far edge) marks nothing.
        const size_t first = (size_t)std::max(std::floor((piece_lo - lo) / width), 0.0);
        const double up = std::ceil((piece_hi - lo) / width);
        size_t last = up > 0.0 ? (size_t)up : 0;
        last = last > 0 ? last - 1 : 0;
        last = std::min(std::max(last, first), (size_t)LINE_MASK_BINS - 1);
        for (size_t b = first; b <= last; ++b) blocked[b] = true;
    }
}

}  // extern "C" (the skyline below holds member templates)

// A skyline query (popup/src/obstacles/skyline.rs:22-38): every arc (azimuth lo, hi, nearest
// range) of an edge near the receiver that may meet the wedge [lo, hi] within the radius.
using SkylineQuery =
    std::function<void(double lo, double hi, double radius, const std::function<void(const double *arc)> &visit)>;

// The receiver skyline over a scene (popup/src/obstacles/skyline.rs:22-110) in the reference's
// frame: steps with y growing south, so scene point (x, y) (y north) is (x, -y); cells of 256
// steps, each edge listed in the cells its supercover walk passes through
// (tiles/src/obstacles/cells.rs:13-47), consecutive edges of an outline in one run, and a cell's
// height the tallest of its outlines (popup/src/obstacles/tile.rs:93-104).
struct SceneSkyline {
    struct Run {
        uint32_t outline, first_edge, count;
    };
    std::unordered_map<uint64_t, std::vector<Run>> runs;
    std::unordered_map<uint64_t, double> tallest;
    static uint64_t key(int64_t column, int64_t row) {
        return ((uint64_t)(uint32_t)(int32_t)column << 32) | (uint64_t)(uint32_t)(int32_t)row;
    }

    // The cells start -> end passes through, 4-connected in walking order; a tie steps the row
    // and the walk never leaves the box of its end cells (cells.rs:13-47).
    template <class Visit>
    static void edge_cells(int64_t sx, int64_t sy, int64_t ex, int64_t ey, Visit visit) {
        const int64_t cs = 256;
        auto div = [](int64_t a, int64_t b) { return a >= 0 ? a / b : -((-a + b - 1) / b); };
        int64_t cell[2] = {div(sx, cs), div(sy, cs)};
        const int64_t last[2] = {div(ex, cs), div(ey, cs)};
        const double delta[2] = {(double)(ex - sx), (double)(ey - sy)};
        const int64_t step[2] = {delta[0] >= 0.0 ? 1 : -1, delta[1] >= 0.0 ? 1 : -1};
        const int64_t start[2] = {sx, sy};
        double t_delta[2], t_max[2];
        for (int axis = 0; axis < 2; ++axis) {
            t_delta[axis] = delta[axis] != 0.0 ? std::fabs((double)cs / delta[axis]) : INF;
            if (delta[axis] == 0.0) {
                t_max[axis] = INF;
            } else {
                const int64_t boundary = (cell[axis] + (delta[axis] >= 0.0 ? 1 : 0)) * cs;
                t_max[axis] = std::fabs((double)(boundary - start[axis]) / delta[axis]);
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

    explicit SceneSkyline(const Scene &s) {
        for (uint32_t o = 0; o < s.outlines.size(); ++o) {
            const qm_outline &rec = s.outlines[o];
            for (uint32_t k = 0; k + 1 < rec.vertex_count; ++k) {
                const size_t e = rec.first_vertex + k;
                edge_cells(s.vertices[2 * e], -(int64_t)s.vertices[2 * e + 1], s.vertices[2 * e + 2],
                           -(int64_t)s.vertices[2 * e + 3], [&](int64_t c, int64_t r) {
                               std::vector<Run> &list = runs[key(c, r)];
                               if (!list.empty() && list.back().outline == o &&
                                   list.back().first_edge + list.back().count == k)
                                   ++list.back().count;
                               else
                                   list.push_back(Run{o, k, 1});
                               double &top = tallest.try_emplace(key(c, r), -INF).first->second;
                               top = std::max(top, (double)rec.height_m);
                           });
            }
        }
    }

    // The arcs for the receiver at scene steps (rx, ry), wedge [lo, hi], radius and sight-line
    // floor: cells beyond the radius or wholly outside the wedge are skipped, so are cells whose
    // tallest outline and walls whose height stay at or under the floor (skyline.rs:39-110).
    void query(const Scene &s, int64_t rx, int64_t ry, double lo, double hi, double radius_m, double floor_m,
               const std::function<void(const double *)> &visit) const {
        const double m = s.step_m, cs = 256.0;
        const double ox = (double)rx, oy = -(double)ry;
        const double low[2] = {std::cos(lo), std::sin(lo)}, high[2] = {std::cos(hi), std::sin(hi)};
        auto relative = [&](size_t v, double out[2]) {
            out[0] = ((double)s.vertices[2 * v] - ox) * m;
            out[1] = (oy + (double)s.vertices[2 * v + 1]) * m;
        };
        const int64_t row0 = (int64_t)std::floor((oy - radius_m / m) / cs);
        const int64_t row1 = (int64_t)std::floor((oy + radius_m / m) / cs);
        const int64_t col0 = (int64_t)std::floor((ox - radius_m / m) / cs);
        const int64_t col1 = (int64_t)std::floor((ox + radius_m / m) / cs);
        for (int64_t row = row0; row <= row1; ++row) {
            const double south = (oy - (double)(row + 1) * cs) * m, north = (oy - (double)row * cs) * m;
            const double dy = std::max(std::max(south, -north), 0.0);
            for (int64_t column = col0; column <= col1; ++column) {
                const double west = ((double)column * cs - ox) * m, east = ((double)(column + 1) * cs - ox) * m;
                const double dx = std::max(std::max(west, -east), 0.0);
                if (dx * dx + dy * dy > radius_m * radius_m) continue;
                const double corners[4][2] = {{west, south}, {east, south}, {west, north}, {east, north}};
                bool below = true, above = true;
                for (const auto &c : corners) {
                    below = below && low[0] * c[1] - low[1] * c[0] < 0.0;
                    above = above && c[0] * high[1] - c[1] * high[0] < 0.0;
                }
                if (below || above) continue;
                const auto found = runs.find(key(column, row));
                if (found == runs.end() || tallest.at(key(column, row)) <= floor_m) continue;
                for (const Run &run : found->second) {
                    const qm_outline &rec = s.outlines[run.outline];
                    if (rec.building == 0 && (double)rec.height_m <= floor_m) continue;
                    const size_t first = rec.first_vertex + run.first_edge;
                    double a[2], b[2];
                    relative(first, a);
                    double azimuth_a = std::atan2(a[1], a[0]);
                    for (size_t next = first + 1; next <= first + run.count; ++next) {
                        relative(next, b);
                        const double azimuth_b = std::atan2(b[1], b[0]);
                        // The edge's nearest point to the receiver (skyline.rs:9-20).
                        const double ex = b[0] - a[0], ey = b[1] - a[1], length2 = ex * ex + ey * ey;
                        const double t =
                            length2 > 0.0 ? std::min(std::max(-(a[0] * ex + a[1] * ey) / length2, 0.0), 1.0) : 0.0;
                        const double px = a[0] + t * ex, py = a[1] + t * ey;
                        const double nearest = std::sqrt(px * px + py * py);
                        if (nearest >= 1e-6 && nearest <= radius_m) {
                            const double unwrapped_b = azimuth_a + line_wrap_to_pi(azimuth_b - azimuth_a);
                            const double arc[3] = {std::min(azimuth_a, unwrapped_b), std::max(azimuth_a, unwrapped_b),
                                                   nearest};
                            visit(arc);
                        }
                        a[0] = b[0];
                        a[1] = b[1];
                        azimuth_a = azimuth_b;
                    }
                }
            }
        }
    }
};

// A query handing over a fixed list of arcs whatever the wedge (the mask re-checks each).
static SkylineQuery listed_arcs(const double *arcs, size_t n_arcs) {
    return [arcs, n_arcs](double, double, double, const std::function<void(const double *)> &visit) {
        for (size_t k = 0; k < n_arcs; ++k) visit(arcs + 3 * k);
    };
}

extern "C" {

// push_wide_bucket_nodes (line.rs:208-315): geometry-placed nodes of a wide bucket with something
// in front of it; nothing otherwise.
static void line_wide_nodes(const LinePiece &g, double angle_lo, double angle_hi, const SkylineQuery &skyline,
                            std::vector<LineNode> &nodes) {
    const double along_lo = g.along_at_angle(angle_lo), along_hi = g.along_at_angle(angle_hi);
    const double azimuth_a = g.azimuth_at(along_lo);
    const double turn = line_wrap_to_pi(g.azimuth_at(along_hi) - azimuth_a);
    const double span = std::fabs(turn);
    if (span < LINE_WIDE_MIN_SPAN) return;
    const double span_lo = turn < 0.0 ? azimuth_a + turn : azimuth_a;
    const double span_hi = turn < 0.0 ? azimuth_a : azimuth_a + turn;
    const double range_lo = g.range_at(along_lo), range_hi = g.range_at(along_hi);
    double a[3], b[3];
    g.point(along_lo, a);
    g.point(along_hi, b);
    const double chord = std::hypot(a[0] - b[0], a[1] - b[1]);
    const double centre_range = g.range_at(g.along_at_angle(0.5 * (angle_lo + angle_hi)));
    const double radius = std::min(std::min(range_lo, range_hi), centre_range) + chord;
    const double width = span / LINE_MASK_BINS;
    bool blocked[LINE_MASK_BINS] = {};
    skyline(span_lo, span_hi, radius,
            [&](const double *arc) { line_mark(g, arc, radius, span_lo, span_hi, width, blocked); });
    bool any = false;
    for (bool v : blocked) any = any || v;
    if (!any) return;
    const double lo_a = std::min(along_lo, along_hi), hi_a = std::max(along_lo, along_hi);
    auto angle_at_azimuth = [&](double azimuth, double fallback) {
        double along;
        if (!g.along_at_azimuth(azimuth, along)) return fallback;
        return g.angle_at(std::min(std::max(along, lo_a), hi_a));
    };
    const double angle_at_span_lo = turn < 0.0 ? angle_hi : angle_lo;
    const double angle_at_span_hi = turn < 0.0 ? angle_lo : angle_hi;
    int bin = 0;
    while (bin < LINE_MASK_BINS) {
        const bool run_blocked = blocked[bin];
        int run_end = bin;
        while (run_end < LINE_MASK_BINS && blocked[run_end] == run_blocked) ++run_end;
        const double run_lo = span_lo + bin * width;
        const double run_hi = run_end == LINE_MASK_BINS ? span_hi : span_lo + run_end * width;
        const int parts = (int)std::min(std::max(std::ceil((run_hi - run_lo) / LINE_PART_MAX_SPAN), 1.0),
                                        (double)LINE_MAX_PARTS);
        const double step = (run_hi - run_lo) / parts;
        for (int part = 0; part < parts; ++part) {
            const double part_lo = run_lo + part * step;
            const double part_hi = (part + 1 == parts && run_end == LINE_MASK_BINS) ? span_hi : part_lo + step;
            const double edge_lo = (bin == 0 && part == 0) ? angle_at_span_lo : angle_at_azimuth(part_lo, angle_at_span_lo);
            const double edge_hi =
                (run_end == LINE_MASK_BINS && part + 1 == parts) ? angle_at_span_hi : angle_at_azimuth(part_hi, angle_at_span_hi);
            double along;
            if (!g.along_at_azimuth(0.5 * (part_lo + part_hi), along)) along = g.along_at_angle(0.5 * (edge_lo + edge_hi));
            nodes.push_back(LineNode{along, std::fabs(edge_hi - edge_lo), run_blocked});
        }
        bin = run_end;
    }
}

// line_quadrature_nodes (line.rs:180-206): one bucket under 3 degrees, else five of equal dphi,
// each its centre node unless it is wide and something stands in front of it.
static void line_nodes(const LinePiece &g, const SkylineQuery &skyline, std::vector<LineNode> &nodes) {
    nodes.clear();
    const double span = g.span();
    const int buckets = span < LINE_ONE_BUCKET_SPAN ? 1 : LINE_BUCKETS;
    const double bucket_angle = span / buckets;
    for (int bucket = 0; bucket < buckets; ++bucket) {
        const double angle_lo = g.angle0 + bucket * bucket_angle, angle_hi = angle_lo + bucket_angle;
        const size_t before = nodes.size();
        line_wide_nodes(g, angle_lo, angle_hi, skyline, nodes);
        if (nodes.size() == before)
            nodes.push_back(LineNode{g.along_at_angle(angle_lo + 0.5 * bucket_angle), angle_hi - angle_lo, true});
    }
}

// A_ground per band over one mean plane (physics/src/cnossos/ground.rs:8-139) for a source at
// (sx, sz) and a receiver at (rx, rz) with the given ground factors and state.
void qmo_ground_attenuation_bands(double slope, double intercept, double sx, double sz, double rx, double rz,
                                  double g_path, double g_impedance, double g_floor, int state, double *out) {
    const EqGeometry g = geometry_over(MeanPlane{slope, intercept}, sx, sz, rx, rz);
    ground_attenuation_bands(g, GroundFactors{g_path, g_impedance, g_floor}, state, out);
}

// ---------------------------------------------------------------------------------------------
// The quantile table of a line of Poisson emitters (Kurze 1971), as the reference generates it
// (physics/src/percentile_tests.rs:1-102, physics/src/percentile.rs:11-21): one SplitMix64 stream
// over the rows in order; per sample a Poisson count of emitters uniform on the simulated length,
// their intensities 1 / (1 + x^2) summed with the mean of those beyond, over the line's mean;
// each row's samples sorted and read at probabilities (k + 0.5) / 100.

namespace {

struct SplitMix64 {  // percentile_tests.rs:5-21
    uint64_t state;
    double uniform() {
        state += 0x9e3779b97f4a7c15ull;
        uint64_t z = state;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return (double)((z ^ (z >> 31)) >> 11) / (double)(1ull << 53);
    }
};

size_t percentile_poisson(SplitMix64 &random, double mean) {  // percentile_tests.rs:34-47
    const double pi = 3.14159265358979323846;
    if (mean > 50.0) {
        const double a = std::sqrt(-2.0 * std::log(1.0 - random.uniform()));
        const double normal = a * std::cos(2.0 * pi * random.uniform());
        return (size_t)std::max(std::round(mean + std::sqrt(mean) * normal), 0.0);
    }
    const double limit = std::exp(-mean);
    size_t count = 0;
    double product = random.uniform();
    while (product > limit) {
        ++count;
        product *= random.uniform();
    }
    return count;
}

}  // namespace

// Rows [0, n_rows) of the table (row r at lambda = 1e-4 * 10^(r / 8)), each QUANTILES = 100
// values rounded to float as the table stores them: table[n_rows][100]. Rows are generated in
// order from the seed, so any row needs the ones before it.
void qmo_percentile_table(int n_rows, float *table) {
    const double pi = 3.14159265358979323846;
    SplitMix64 random{0x5eed1971ull};
    std::vector<double> samples;
    for (int row = 0; row < n_rows; ++row) {
        const double lambda = 1e-4 * std::pow(10.0, (double)row / 8.0);
        const double half_length = std::max(5.0 / lambda, 200.0);            // percentile_tests.rs:31-33
        const size_t count = (size_t)std::min(20000.0 * std::max(0.01 / lambda, 1.0), 1000000.0);
        const double mean_inside = lambda * 2.0 * half_length;
        const double outside = lambda * 2.0 * (pi / 2.0 - std::atan(half_length));
        const double mean = lambda * pi;
        samples.resize(count);
        for (size_t i = 0; i < count; ++i) {
            const size_t emitters = percentile_poisson(random, mean_inside);
            double inside = 0.0;
            for (size_t e = 0; e < emitters; ++e) {
                const double x = (2.0 * random.uniform() - 1.0) * half_length;
                inside += 1.0 / (1.0 + x * x);
            }
            samples[i] = (inside + outside) / mean;
        }
        std::sort(samples.begin(), samples.end());
        for (int k = 0; k < 100; ++k)
            table[row * 100 + k] = (float)samples[(size_t)(((double)k + 0.5) / 100.0 * (double)count)];
    }
}

// The sampler over that table (physics/src/percentile.rs:27-160): the intensity, relative to its
// mean, that a line of `lambda` emitters per distance stays below with probability p.

namespace {

const float *percentile_rows() {  // the 41 x 100 table, from the simulation above, made once
    static const std::vector<float> table = [] {
        std::vector<float> t(41 * 100);
        qmo_percentile_table(41, t.data());
        return t;
    }();
    return table.data();
}

// The standard normal quantile by Acklam's rational approximation (percentile.rs:27-71).
double normal_quantile(double p) {
    static const double A[6] = {-3.969683028665376e1, 2.209460984245205e2, -2.759285104469687e2,
                                1.38357751867269e2,   -3.066479806614716e1, 2.506628277459239};
    static const double B[5] = {-5.447609879822406e1, 1.615858368580409e2, -1.556989798598866e2,
                                6.680131188771972e1, -1.328068155288572e1};
    static const double C[6] = {-7.784894002430293e-3, -3.223964580411365e-1, -2.400758277161838,
                                -2.549671010366478,    4.374664141464968,     2.938163982698783};
    static const double D[4] = {7.784695709041462e-3, 3.224671290700398e-1, 2.445134137142996, 3.754408661907416};
    auto tail = [&](double q) {
        return (((((C[0] * q + C[1]) * q + C[2]) * q + C[3]) * q + C[4]) * q + C[5]) /
               ((((D[0] * q + D[1]) * q + D[2]) * q + D[3]) * q + 1.0);
    };
    if (p < 0.02425) return tail(std::sqrt(-2.0 * std::log(p)));
    if (p > 1.0 - 0.02425) return -tail(std::sqrt(-2.0 * std::log(1.0 - p)));
    const double q = p - 0.5, r = q * q;
    return (((((A[0] * r + A[1]) * r + A[2]) * r + A[3]) * r + A[4]) * r + A[5]) * q /
           (((((B[0] * r + B[1]) * r + B[2]) * r + B[3]) * r + B[4]) * r + 1.0);
}

double quantile_probability(int k) { return ((double)k + 0.5) / 100.0; }

double relative_intensity(double lambda, double p) {
    const double pi = 3.14159265358979323846, lambda_min = 1e-4;
    if (!std::isfinite(lambda)) return 1.0;
    if (lambda <= 0.0) return 0.0;
    const double bottom = quantile_probability(0), top = quantile_probability(99);
    auto passing = [&](double ln_p) {  // percentile.rs:77-80
        const double s = -ln_p / (2.0 * lambda);
        return 1.0 / (lambda * pi * (1.0 + s * s));
    };
    if (lambda >= 10.0) {  // percentile.rs:83-86: a dense line is normal
        const double deviation = 1.0 / std::sqrt(2.0 * pi * lambda);
        return std::max(1.0 + deviation * normal_quantile(std::min(std::max(p, bottom), top)), 0.0);
    }
    if (p > top) return relative_intensity(lambda, top) + passing(std::log(p)) - passing(std::log(top));
    if (lambda < lambda_min) return lambda / lambda_min * relative_intensity(lambda_min, p);
    // table_position (percentile.rs:89-93)
    const double position = std::min(std::max(std::log10(lambda / lambda_min) * 8.0, 0.0), 40.0);
    const int row = (int)std::floor(position);
    const double fraction = position - std::trunc(position);
    // quantile_position (percentile.rs:97-104)
    const double pq = std::max(p, bottom);
    const int k = std::min((int)std::floor(pq * 100.0 - 0.5), 98);
    const double t = (std::log(1.0 - pq) - std::log(1.0 - quantile_probability(k))) /
                     (std::log(1.0 - quantile_probability(k + 1)) - std::log(1.0 - quantile_probability(k)));
    const float *table = percentile_rows();
    auto log_quantile = [&](int r) {  // percentile.rs:107-114
        const double here = std::log(std::max((double)table[r * 100 + k], 1e-30));
        const double next = std::log(std::max((double)table[r * 100 + k + 1], 1e-30));
        return here + t * (next - here);
    };
    const double low = log_quantile(row), high = log_quantile(std::min(row + 1, 40));
    return std::exp(low + fraction * (high - low));
}

}  // namespace

// relative_intensity at n probabilities for one lambda: out[n].
void qmo_relative_intensities(double lambda, const double *p, size_t n, double *out) {
    for (size_t i = 0; i < n; ++i) out[i] = relative_intensity(lambda, p[i]);
}

// ---------------------------------------------------------------------------------------------
// The state rays and the rubber band on their own (physics/src/cnossos/rubber_band.rs), for the
// reference's rubber-band tests. Points are (x, z) pairs; state 0 homogeneous, 1 favourable; a
// radius_m <= 0 takes the state ray between source and receiver (`StateRay::between`).

static StateRay rb_ray(int state, double radius_m, const double *source, const double *receiver) {
    StateRay ray = StateRay::between(state, PP{source[0], source[1]}, PP{receiver[0], receiver[1]});
    if (radius_m > 0.0) ray.radius = radius_m;
    return ray;
}

double qmo_path_difference(int state, double radius_m, const double *source, const double *receiver,
                           const double *from, const double *points, size_t n, const double *to) {
    const StateRay ray = rb_ray(state, radius_m, source, receiver);
    std::vector<PP> p(n);
    for (size_t k = 0; k < n; ++k) p[k] = PP{points[2 * k], points[2 * k + 1]};
    return ray.path_difference(PP{from[0], from[1]}, p.data(), n, PP{to[0], to[1]});
}

// diffraction_path: returns whether the direct ray is blocked; the band's points (up to cap) and
// the blocking candidates (up to cap), with their counts.
int qmo_diffraction_path(int state, double radius_m, const double *source, const double *receiver,
                         const double *candidates, size_t n, double *points, size_t *n_points, double *blocking,
                         size_t *n_blocking, size_t cap) {
    const StateRay ray = rb_ray(state, radius_m, source, receiver);
    std::vector<PP> c(n), out;
    for (size_t k = 0; k < n; ++k) c[k] = PP{candidates[2 * k], candidates[2 * k + 1]};
    std::vector<Blocking> block, hull;
    bool blocked = false;
    diffraction_path(ray, PP{source[0], source[1]}, PP{receiver[0], receiver[1]}, c, block, hull, out, blocked);
    *n_points = out.size();
    for (size_t k = 0; k < out.size() && k < cap; ++k) {
        points[2 * k] = out[k].x;
        points[2 * k + 1] = out[k].z;
    }
    *n_blocking = block.size();
    for (size_t k = 0; k < block.size() && k < cap; ++k) {
        blocking[2 * k] = block[k].x;
        blocking[2 * k + 1] = block[k].z;
    }
    return blocked ? 1 : 0;
}

// The state's ray from a to b at x: the chord's altitude plus the arc's sag.
double qmo_state_ray_altitude(int state, double radius_m, const double *source, const double *receiver,
                              const double *a, const double *b, double x) {
    const StateRay ray = rb_ray(state, radius_m, source, receiver);
    const PP pa{a[0], a[1]}, pb{b[0], b[1]};
    return chord_altitude(pa, pb, x) + ray.sag(pa, pb).at(x - pa.x);
}

// The geometry of a piece: out = (length, perpendicular, subtended angle, divergence factor);
// -1 for a piece shorter than a millimetre.
int qmo_line_geometry(const double *start, const double *end, double *out) {
    LinePiece g;
    if (!g.make(start, end)) return -1;
    out[0] = g.length;
    out[1] = g.perp;
    out[2] = g.span();
    out[3] = g.divergence();
    return 0;
}

// One straight line piece of a source at one receiver: `source_rays` for a line and `add_ray`
// (popup/src/evaluate.rs:215-265, 118-152). The piece runs from a to b (steps, anywhere); its
// ends stand on the terrain there plus the source's height; its quadrature nodes
// (`line_nodes`, over the skyline query given) each send a ray from their point along the piece,
// over the obstacles only where the mask says they can stand, weighted by the node's angle times
// the line's divergence. `src.energy` is the power per metre of the piece.
static int evaluate_line_piece(const Scene &s, const Receiver &r, const double a[2], const double b[2],
                               const qm_source &src, const SkylineQuery &skyline, Worker &w, PairResult &out) {
    for (int period = 0; period < PERIODS; ++period) {
        for (int b2 = 0; b2 < BANDS; ++b2) out.bands[period][b2] = 0.0;
        for (int st = 0; st < 2; ++st) out.states[st][period] = 0.0;
    }
    double za, zb, ga, gb;
    terrain_at(s, a[0], a[1], za, ga);
    terrain_at(s, b[0], b[1], zb, gb);
    const double start[3] = {(a[0] - (double)r.x) * s.step_m, (a[1] - (double)r.y) * s.step_m,
                             za + src.height_m - r.altitude_m};
    const double end[3] = {(b[0] - (double)r.x) * s.step_m, (b[1] - (double)r.y) * s.step_m,
                           zb + src.height_m - r.altitude_m};
    LinePiece g;
    if (!g.make(start, end)) return 0;
    std::vector<LineNode> nodes;
    line_nodes(g, skyline, nodes);
    const double divergence = g.divergence();
    const double to[2] = {(double)r.x, (double)r.y};
    for (const LineNode &node : nodes) {
        const double fraction = node.along / g.length;
        const double point[2] = {a[0] + fraction * (b[0] - a[0]), a[1] + fraction * (b[1] - a[1])};
        fill_profile(s, point, to, w.profile);
        w.crossings.clear();
        if (node.on_ray) {
            scene_crossings(s, point, to, w.crossings);
            if (r.own_footprint != 0) {
                size_t kept = 0;
                for (size_t i = 0; i < w.crossings.size(); ++i)
                    if (w.crossings[i].footprint_id != r.own_footprint) w.crossings[kept++] = w.crossings[i];
                w.crossings.resize(kept);
            }
        }
        const double azimuth = std::atan2(((double)r.y - point[1]) * s.step_m, ((double)r.x - point[0]) * s.step_m);
        double p[PERIODS];
        for (int period = 0; period < PERIODS; ++period) p[period] = favourable_at(s.favourable[period], azimuth);
        RayEnds ends;
        ends.source_height_m = src.height_m;
        ends.has_source_ground = false;
        ends.source_ground_m = 0.0;
        ends.receiver_altitude_m = r.altitude_m;
        ends.has_source_ground_factor = src.ground_factor >= 0.0f;
        ends.source_ground_factor = src.ground_factor;
        ends.platform_half_width_m = src.platform_half_width_m;
        ends.own_footprint = src.footprint_id;
        Transfer transfer;
        StateBoundary boundaries[2];
        ray_terms(w.profile, w.crossings, ends, p, s.alpha, w.ray, transfer, boundaries, true);
        const double weight = node.weight * divergence;
        for (int period = 0; period < PERIODS; ++period)
            for (int band = 0; band < BANDS; ++band) {
                const double power = weight * (double)src.energy[period][band];
                out.bands[period][band] += power * transfer.periods[period][band];
                out.states[0][period] += power * transfer.states[0][band];
                out.states[1][period] += power * transfer.states[1][band];
            }
    }
    return (int)nodes.size();
}

// A line piece's received energy at a receiver (a lattice point at receiver_altitude_m, with its
// own footprint): bands[3][8], states[2][3]; returns the number of quadrature nodes. With
// scene_skyline the nodes see the scene's own skyline from the receiver, its floor the source's
// height and never under the ground (popup/src/evaluate.rs:225-242); otherwise the arcs listed.
int qmo_line_piece(void *scene, const int64_t receiver[2], double receiver_altitude_m, uint64_t own_footprint,
                   const double a[2], const double b[2], const qm_source *source, int scene_skyline,
                   const double *arcs, size_t n_arcs, double *bands, double *states) {
    const Scene &s = *static_cast<Scene *>(scene);
    const Receiver r{receiver[0], receiver[1], receiver_altitude_m, own_footprint};
    Worker w;
    PairResult out;
    int n;
    if (scene_skyline) {
        const SceneSkyline sky(s);
        const double floor_m = std::max((double)source->height_m, 0.0);
        const SkylineQuery query = [&](double lo, double hi, double radius,
                                       const std::function<void(const double *)> &visit) {
            sky.query(s, r.x, r.y, lo, hi, radius, floor_m, visit);
        };
        n = evaluate_line_piece(s, r, a, b, *source, query, w, out);
    } else {
        n = evaluate_line_piece(s, r, a, b, *source, listed_arcs(arcs, n_arcs), w, out);
    }
    for (int period = 0; period < PERIODS; ++period) {
        for (int band = 0; band < BANDS; ++band) bands[period * BANDS + band] = out.bands[period][band];
        for (int st = 0; st < 2; ++st) states[st * PERIODS + period] = out.states[st][period];
    }
    return n;
}

// The skyline arcs (azimuth lo, hi, nearest range; metres east and north of the receiver) that a
// receiver at scene steps `receiver` gets for the wedge [lo, hi] within radius_m above floor_m,
// once per cell an edge is listed in (popup/src/obstacles/skyline.rs:39-110). Writes at most
// `cap` arcs; returns how many there are.
size_t qmo_skyline_arcs(void *scene, const int64_t receiver[2], double lo, double hi, double radius_m, double floor_m,
                        double *out, size_t cap) {
    const Scene &s = *static_cast<Scene *>(scene);
    const SceneSkyline sky(s);
    size_t n = 0;
    sky.query(s, receiver[0], receiver[1], lo, hi, radius_m, floor_m, [&](const double *arc) {
        if (n < cap)
            for (int k = 0; k < 3; ++k) out[3 * n + k] = arc[k];
        ++n;
    });
    return n;
}

// The quadrature nodes of a piece (start, end: metres relative to the receiver) with each wide
// bucket querying the scene's skyline from the receiver at scene steps `receiver` above floor_m,
// as the line evaluation does (popup/src/evaluate.rs:225-242); up to cap written. Returns the
// count, -1 for a degenerate piece.
int qmo_scene_line_nodes(void *scene, const int64_t receiver[2], double floor_m, const double *start,
                         const double *end, double *along, double *weight, uint8_t *on_ray, size_t cap) {
    const Scene &s = *static_cast<Scene *>(scene);
    LinePiece g;
    if (!g.make(start, end)) return -1;
    const SceneSkyline sky(s);
    const SkylineQuery query = [&](double lo, double hi, double radius, const std::function<void(const double *)> &visit) {
        sky.query(s, receiver[0], receiver[1], lo, hi, radius, floor_m, visit);
    };
    std::vector<LineNode> nodes;
    line_nodes(g, query, nodes);
    for (size_t k = 0; k < nodes.size() && k < cap; ++k) {
        along[k] = nodes[k].along;
        weight[k] = nodes[k].weight;
        on_ray[k] = nodes[k].on_ray ? 1 : 0;
    }
    return (int)nodes.size();
}

double qmo_line_in_plane_angle_at(const double *start, const double *end, double along) {
    LinePiece g;
    return g.make(start, end) ? g.angle_at(along) : NAN;
}

// The quadrature nodes of a piece given the arcs a skyline query hands over (arcs[n][3]: azimuth
// lo, hi, nearest horizontal range); up to cap written. Returns the count, -1 for a degenerate
// piece. The mask re-checks each arc's range and span; which edges become arcs (their heights
// against the source's, popup/src/obstacles/skyline.rs:22-110) is the caller's choice.
int qmo_line_nodes(const double *start, const double *end, const double *arcs, size_t n_arcs, double *along,
                   double *weight, uint8_t *on_ray, size_t cap) {
    LinePiece g;
    if (!g.make(start, end)) return -1;
    std::vector<LineNode> nodes;
    line_nodes(g, listed_arcs(arcs, n_arcs), nodes);
    for (size_t k = 0; k < nodes.size() && k < cap; ++k) {
        along[k] = nodes[k].along;
        weight[k] = nodes[k].weight;
        on_ray[k] = nodes[k].on_ray ? 1 : 0;
    }
    return (int)nodes.size();
}

// p of one period's row for sound travelling along azimuth_rad (atan2(north, east)): the scene's
// favourable row (float) interpolated between sector centres (physics/src/weather.rs:61-70).
double qmo_favourable_at(const float *row, double azimuth_rad) { return favourable_at(row, azimuth_rad); }

uint32_t qmo_level_bin(double level, double level_min, double bin_db, uint32_t n_bins) {
    return level_bin(level, level_min, bin_db, n_bins);
}

// Map cells. `cell` (paint/src/levels.rs:25-33): 80 + 20 log2(sone), silence (254) when NaN or
// below 0, else rounded half away from zero and capped at 253.
uint8_t qmo_nden_cell(double sone) {
    const double byte = 80.0 + 20.0 * std::log2(sone);
    if (std::isnan(byte) || byte < 0.0) return 254;
    return (uint8_t)std::min(std::round(byte), 253.0);
}

// `lden_cell` (paint/src/levels.rs:87-98): -1 for an energy that is negative or not finite (the
// reference's error), 254 below 1, else round(2 level_db) capped at 253, level_db = 10 log10
// (physics/src/bands.rs:45-56).
int qmo_lden_cell(double energy) {
    if (!std::isfinite(energy) || energy < 0.0) return -1;
    if (energy < 1.0) return 254;
    return (int)std::min(std::round(2.0 * (10.0 * std::log10(energy))), 253.0);
}

// HM3 streams. `paeth_prediction` (paint/src/hm3.rs:68-93): PNG filter 4 over a 512-wide tile,
// zeros outside it, ties to left, then above.
static uint8_t hm3_paeth(const uint8_t *cells, size_t at) {
    const size_t P = QM_HM3_TILE_PX;
    const bool has_left = at % P != 0, has_above = at >= P;
    const int left = has_left ? cells[at - 1] : 0;
    const int above = has_above ? cells[at - P] : 0;
    const int corner = has_left && has_above ? cells[at - P - 1] : 0;
    const int estimate = left + above - corner;
    const int dl = std::abs(estimate - left), da = std::abs(estimate - above), dc = std::abs(estimate - corner);
    if (dl <= da && dl <= dc) return (uint8_t)left;
    return (uint8_t)(da <= dc ? above : corner);
}

// `encode_metric_tile` up to its Brotli stage (paint/src/hm3.rs:95-109): header ("HM3 \x07" or
// "HMD \x01", hm3.rs:22-27), layer byte, residuals. Returns 0, or -1 for a layer above QM_LAYERS.
int qmo_hm3_predict(const uint8_t *cells, uint8_t layer, int metric, uint8_t *stream) {
    if (layer > QM_LAYERS) return -1;
    static const uint8_t header[2][5] = {{'H', 'M', '3', ' ', 0x07}, {'H', 'M', 'D', ' ', 0x01}};
    std::memcpy(stream, header[metric ? 1 : 0], 5);
    stream[5] = layer;
    const size_t n = (size_t)QM_HM3_TILE_PX * QM_HM3_TILE_PX;
    for (size_t at = 0; at < n; ++at) stream[6 + at] = (uint8_t)(cells[at] - hm3_paeth(cells, at));
    return 0;
}

// The residuals' inverse, as `decode_metric_tile` applies it after Brotli (paint/src/hm3.rs:
// 162-165): in place, in order, each byte plus the prediction from the bytes already restored.
void qmo_hm3_unpredict(uint8_t *residuals) {
    const size_t n = (size_t)QM_HM3_TILE_PX * QM_HM3_TILE_PX;
    for (size_t at = 0; at < n; ++at) residuals[at] = (uint8_t)(residuals[at] + hm3_paeth(residuals, at));
}

// `PaintedCells::from_painted` (paint/src/levels.rs:55-68) with `lden_cells` (:100-111) and
// `cells_of` (:36-38) over n pixels: lden_cells[n][7] from lden_energy[n][6], nden_cells[n][7]
// from sone[n][7] (both skipped when sone is null), 255 for unassessed pixels (assessed null: all
// assessed). Returns -1, or pixel * 8 + layer of the first invalid energy in pixel order (layer 6:
// the total, the layers summed in order), after which the outputs are not meaningful.
int64_t qmo_quantize_cells(const double *lden_energy, const double *sone, const uint8_t *assessed, size_t n,
                           uint8_t *lden_cells, uint8_t *nden_cells) {
    constexpr int L = QM_LAYERS, W = QM_LAYERS + 1;
    for (size_t p = 0; p < n; ++p) {
        if (assessed && assessed[p] == 0) {
            for (int l = 0; l < W; ++l) {
                lden_cells[p * W + l] = 255;
                if (sone) nden_cells[p * W + l] = 255;
            }
            continue;
        }
        double total = 0.0;
        for (int l = 0; l < L; ++l) {
            const double e = lden_energy[p * L + l];
            const int c = qmo_lden_cell(e);
            if (c < 0) return (int64_t)(p * 8 + l);
            lden_cells[p * W + l] = (uint8_t)c;
            total += e;
        }
        const int c = qmo_lden_cell(total);
        if (c < 0) return (int64_t)(p * 8 + L);
        lden_cells[p * W + L] = (uint8_t)c;
        if (sone)
            for (int l = 0; l < W; ++l) nden_cells[p * W + l] = qmo_nden_cell(sone[p * W + l]);
    }
    return -1;
}

// Surrogate training samples (the features of include/qm_surrogate.h and the exact A_boundary of
// the homogeneous state as the label) for cells [cell_begin, cell_end) of a grid against its
// source range: row (cell - cell_begin) * n_src + (source - source_begin). The roofs are the
// vertical path's after clip_roofs_in_closing_order (physics/src/ray.rs:389-404); a path is
// eligible when every obstacle top is a roof-bounding hit, every hit pairs into a roof and at
// most 16 hits (8 roofs) are crossed.
void qmo_surrogate_samples(void *scene, const qm_grid_desc *grid, uint32_t cell_begin, uint32_t cell_end,
                           double *features, double *labels, uint8_t *eligible, int threads) {
    const Scene &s = *static_cast<Scene *>(scene);
    uint32_t sb = grid->source_begin, se = grid->source_end;
    if (se <= sb) {
        sb = 0;
        se = (uint32_t)s.sources.size();
    }
    const uint32_t n_src = se - sb;
    const bool terrain = s.dem_nx != 0;
    std::vector<Worker> workers(std::max(threads, 1));
    parallel_for(cell_end - cell_begin, threads, [&](size_t k, int t) {
        uint32_t cell = cell_begin + (uint32_t)k;
        int64_t x = grid->origin[0] + (int64_t)(cell % grid->nx) * grid->spacing;
        int64_t y = grid->origin[1] + (int64_t)(cell / grid->nx) * grid->spacing;
        Receiver r = make_receiver(s, x, y, grid->height_m, enclosing_building(s, x, y));
        Worker &w = workers[t];
        for (uint32_t si = sb; si < se; ++si) {
            const qm_source &src = s.sources[si];
            size_t row = (k * n_src + (si - sb)) * (terrain ? 2 : 1);
            int64_t from[2] = {src.x, src.y}, to[2] = {r.x, r.y};
            fill_profile(s, from, to, w.profile);
            scene_crossings(s, from, to, w.crossings);
            if (r.own_footprint != 0) {
                size_t kept = 0;
                for (size_t i = 0; i < w.crossings.size(); ++i)
                    if (w.crossings[i].footprint_id != r.own_footprint) w.crossings[kept++] = w.crossings[i];
                w.crossings.resize(kept);
            }
            RayEnds ends;
            ends.source_height_m = src.height_m;
            ends.has_source_ground = false;
            ends.source_ground_m = 0.0;
            ends.receiver_altitude_m = r.altitude_m;
            ends.has_source_ground_factor = src.ground_factor >= 0.0f;
            ends.source_ground_factor = src.ground_factor;
            ends.platform_half_width_m = src.platform_half_width_m;
            ends.own_footprint = src.footprint_id;
            double p[PERIODS] = {0.0, 0.0, 0.0};
            Transfer transfer;
            StateBoundary boundaries[2];
            ray_terms(w.profile, w.crossings, ends, p, s.alpha, w.ray, transfer, boundaries, terrain);
            const PathBuffers &pb = w.ray.pb;
            if (terrain) {
                terrain_sample(s, src, r, w, pb, boundaries, features + row * 32, labels + row * BANDS,
                               eligible + row);
                continue;
            }
            for (int b = 0; b < BANDS; ++b) labels[row * BANDS + b] = boundaries[0].attenuation[b];
            // Eligibility: tops all roof-bounding, hits all paired, at most 16 hits.
            bool ok = pb.tops.size() == pb.buildings.size() && pb.buildings.size() <= 16;
            for (size_t a = 0; a < pb.buildings.size() && ok;) {
                size_t e = a;
                while (e < pb.buildings.size() && pb.buildings[e].id == pb.buildings[a].id) ++e;
                if ((e - a) % 2 != 0) ok = false;
                a = e;
            }
            eligible[row] = ok ? 1 : 0;
            double zs, gs, zr, gr, zm, gm;
            terrain_at_point(s, src.x, src.y, zs, gs);
            terrain_at_point(s, r.x, r.y, zr, gr);
            terrain_at_point(s, (src.x + r.x) / 2, (src.y + r.y) / 2, zm, gm);
            double L = std::max(w.profile.horizontal_m, 1.0);
            double *f = features + row * 32;
            f[0] = L / 1000.0;
            f[1] = src.height_m / 10.0;
            f[2] = (r.altitude_m - zr) / 10.0;
            f[3] = (zr - zs) / 10.0;
            f[4] = 0.0;
            f[5] = src.ground_factor >= 0.0f ? (double)src.ground_factor : gs;
            f[6] = gm;
            f[7] = gr;
            for (int q = 0; q < 8; ++q) {
                bool present = q < (int)pb.roofs.size();
                const Roof *rf = present ? &pb.roofs[q] : nullptr;
                f[8 + 3 * q] = present ? rf->x0 / L : 0.0;
                f[9 + 3 * q] = present ? rf->x1 / L : 0.0;
                f[10 + 3 * q] = present ? ((rf->top0 + rf->top1) / 2.0 - zs) / 10.0 : 0.0;
            }
        }
    });
}


// A receiver's horizons for aircraft screening (popup/src/aircraft/horizons.rs:145-198
// Horizons::build) on this scene, laid out as write_f32 lays them out (horizons.rs:50-64, 196-201):
// per point (x, y in steps, fractional allowed), its altitude (m) and the footprint it stands in (0
// none). Terrain: 32 sectors x 48 samples from 30 m to 8 km growing geometrically, a sample outside
// the DEM is no terrain (a flat scene's ground is everywhere); buildings: 256 sectors, a 512 m ray
// each, every building crossing but the point's own footprint's walls and those within 1 cm.
void qmo_flight_horizons(void *scene, const double *xy, const double *altitude_m, const uint64_t *own,
                         size_t n, float *out, int threads) {
    const Scene &s = *static_cast<Scene *>(scene);
    constexpr int BANDS = 6, TSECT = 32, BSECT = 256, SAMPLES = 48;
    const double terrain_limits[BANDS] = {500.0, 1000.0, 2000.0, 3500.0, 5500.0, 8000.0};
    const double building_limits[BANDS] = {16.0, 32.0, 64.0, 128.0, 256.0, 512.0};
    const double tau = 6.283185307179586;
    const double growth = std::pow(8000.0 / 30.0, 1.0 / (double)(SAMPLES - 1));
    const size_t floats = 1 + TSECT * (1 + 2 * BANDS) + 1 + BSECT * (1 + 2 * BANDS);
    struct Edge {
        bool set = false;
        double range = 0.0, tangent = 0.0;
    };
    auto band_of = [&](double range, const double *limits) {
        for (int k = 0; k < BANDS; ++k)
            if (range <= limits[k] + 0.5) return k;
        return BANDS - 1;
    };
    // SectorEdges::write_f32 of one horizon.
    auto write = [&](float *at, int sectors, const std::vector<Edge> &edges, const std::vector<double> &steepest,
                     double all) {
        at[0] = (float)all;
        for (int k = 0; k < sectors; ++k) {
            float *e = at + 1 + k * (1 + 2 * BANDS);
            e[0] = (float)steepest[k];
            for (int b = 0; b < BANDS; ++b) {
                const Edge &edge = edges[k * BANDS + b];
                e[1 + 2 * b] = edge.set ? (float)edge.range : NAN;
                e[2 + 2 * b] = edge.set ? (float)edge.tangent : NAN;
            }
        }
    };
    const bool dem = s.dem_nx != 0;
    const double dem_x1 = dem ? (double)(s.dem_ox + (int64_t)(s.dem_nx - 1) * s.dem_spacing) : 0.0;
    const double dem_y1 = dem ? (double)(s.dem_oy + (int64_t)(s.dem_ny - 1) * s.dem_spacing) : 0.0;
    parallel_for(n, threads, [&](size_t i, int) {
        const double px = xy[2 * i], py = xy[2 * i + 1], alt = altitude_m[i];
        float *o = out + i * floats;
        // Terrain (horizons.rs:154-173)
        std::vector<Edge> te(TSECT * BANDS);
        std::vector<double> ts(TSECT, -INFINITY);
        double tall = -INFINITY;
        for (int k = 0; k < TSECT; ++k) {
            const double angle = ((double)k + 0.5) * tau / (double)TSECT;
            const double dx = std::cos(angle), dy = std::sin(angle);
            double range = 30.0;
            for (int j = 0; j < SAMPLES; ++j) {
                const double qx = px + dx * range / s.step_m, qy = py + dy * range / s.step_m;
                const bool inside = !dem || (qx >= (double)s.dem_ox && qx <= dem_x1 && qy >= (double)s.dem_oy && qy <= dem_y1);
                if (inside) {
                    double z, g;
                    terrain_at(s, qx, qy, z, g);
                    const double tangent = (z - alt) / range;
                    Edge &slot = te[k * BANDS + band_of(range, terrain_limits)];
                    if (!slot.set || tangent > slot.tangent) slot = Edge{true, range, tangent};
                    ts[k] = std::max(ts[k], tangent);
                    tall = std::max(tall, tangent);
                }
                range *= growth;
            }
        }
        write(o, TSECT, te, ts, tall);
        // Buildings (horizons.rs:174-196)
        std::vector<Edge> be(BSECT * BANDS);
        std::vector<double> bs(BSECT, -INFINITY);
        double ball = -INFINITY;
        std::vector<Crossing> crossings;
        const double reach = 512.0;
        for (int k = 0; k < BSECT; ++k) {
            const double angle = ((double)k + 0.5) * tau / (double)BSECT;
            const double dx = std::cos(angle), dy = std::sin(angle);
            const double from[2] = {px, py}, to[2] = {px + dx * reach / s.step_m, py + dy * reach / s.step_m};
            scene_crossings(s, from, to, crossings);
            for (const Crossing &c : crossings) {
                if (!c.building || c.footprint_id == own[i]) continue;
                const double range = c.t * reach;
                if (range <= 0.01) continue;
                double z, g;
                terrain_at(s, px + dx * range / s.step_m, py + dy * range / s.step_m, z, g);
                const double tangent = (z + c.height_m - alt) / range;
                Edge &slot = be[k * BANDS + band_of(range, building_limits)];
                if (!slot.set || tangent > slot.tangent) slot = Edge{true, range, tangent};
                bs[k] = std::max(bs[k], tangent);
                ball = std::max(ball, tangent);
            }
        }
        write(o + 1 + TSECT * (1 + 2 * BANDS), BSECT, be, bs, ball);
    });
}

}  // extern "C"
